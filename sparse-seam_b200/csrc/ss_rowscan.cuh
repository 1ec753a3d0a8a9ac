// ss_rowscan.cuh -- warp-per-tile tile pass and list-driven resolve pass for
// T = 32 (the reference's reported tile size).
//
// Observation the design rests on: a pixel with both a strictly greater and a
// strictly smaller 8-neighbour ("decided" pixel) is in neither mask, and
// neither is any pixel of its flat zone (the zone's flags are the OR of its
// pixels').  On natural images most pixels are decided, so only the others
// need connectivity:
//
//   phase A  row scan, lane = column, one warp instruction per 32 pixels:
//            greater / smaller flags from sliding 3 x 3 row maxima / minima
//            (outside pixels are -1, ignored by a signed max and an unsigned
//            min); decided pixels get both masks 0 at once; the others are
//            appended, in pixel order, to a per-warp list (ballot + popc);
//   phase C  dense over the list: the 8 neighbours of each listed pixel give
//            its flags, whether an equal neighbour lies outside the tile
//            (seam), whether an equal neighbour inside the tile is decided
//            (then the zone is decided too: "dead"), and its links: the first
//            equal listed predecessor (up, up-left, up-right, left) becomes
//            its parent and the left and up-right edges are united
//            (Komura-style equivalence, as the reference's tile labelling,
//            harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:213-281);
//   phase D  flatten; each listed pixel ORs its flags into its root;
//   phase E  in pixel order: live seam zones (touching a seam, flags not
//            both set) get fragment records 0..k-1; listed pixels of the
//            other zones get their masks; the pixels of live seam zones are
//            logged as runs for the resolve pass;
//   phase F  border records: the fragment record of each border pixel, or
//            kDeadRecord when its zone is decided.
//
// Seam merging is wait-free: each pair of tiles joined by equal pixels owns a
// counter and the second tile to arrive unites the pair's live fragments, or
// ORs "both flags" into a live fragment whose partner across the seam is
// dead.  The resolve pass looks up every live fragment's component flags and
// writes the logged runs, so every mask byte is written exactly once.
#pragma once

#include "ss_device.cuh"

namespace ss {

namespace rowscan {

constexpr int T = 32;
constexpr int kSlots = 4 * T;          // fragment slots per tile
constexpr int kPendingCap = T * T;     // logged pixels per tile
constexpr uint8_t kDeadRecord = 0xFE;  // border record of a decided zone
constexpr uint8_t kNoRecord = 0xFF;    // border pixel of a zone inside the tile

// Run-log entry: bits 0-7 record, 8-13 x, 14-19 y, 20-26 length.
__device__ __forceinline__ uint32_t pending_entry(int rec, int x, int y,
                                                  int len) {
    return static_cast<uint32_t>(rec) | (static_cast<uint32_t>(x) << 8) |
           (static_cast<uint32_t>(y) << 14) |
           (static_cast<uint32_t>(len) << 20);
}

// Per-pixel shared word: bits 0-9 parent, 10-12 zone flags (at roots),
// 13-20 record + 1 (at roots of live seam zones), 21-23 own flags.
constexpr uint32_t kParMask = 0x3FFu;
constexpr int kZoneShift = 10;
constexpr int kRecShift = 13;
constexpr int kOwnShift = 21;
constexpr uint32_t kDead = kHasGreater | kHasSmaller;

constexpr int kHaloW = T + 2;   // staged tile rows: columns x0-1 .. x0+T

struct __align__(16) WarpSmem {
    uint32_t word[T * T];
    uint16_t list[T * T];      // listed (undecided) pixels, in pixel order
    uint32_t listed[T];        // per row: listed pixels
    int16_t img[kHaloW * kHaloW];  // tile + halo, -1 outside the image
    uint8_t final_flags[kSlots];
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

// Pixel (gx, gy) of the image, or -1 outside it.
__device__ __forceinline__ int pixel_at(const uint8_t* __restrict__ img,
                                        int64_t pitch, int width, int height,
                                        int gx, int gy) {
    return (static_cast<unsigned>(gx) < static_cast<unsigned>(width) &&
            static_cast<unsigned>(gy) < static_cast<unsigned>(height))
               ? static_cast<int>(__ldg(img + gy * pitch + gx))
               : -1;
}

// Find with path halving.  Used while linking (phase C), when a non-root
// word changes only in its parent bits: halving rewrites those bits with an
// ancestor, which is safe under concurrent linking and halving.
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

// Links the larger root below the smaller one (CAS on the whole word; a
// concurrent OR into the word's flag bits only makes the CAS retry).
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
    // Staged row r holds image row y0 - 1 + r, columns x0 - 1 .. x0 + T
    // (staged column c = image column x0 - 1 + c); -1 outside the image.  All
    // loads are issued before the first store so they overlap.
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

    // -- phase A: flags, decided pixels, list ---------------------------------
    const bool col_ok = lane < g.tw;
    const int16_t* scol = sm.img + lane;   // staged column lane - 1 .. lane + 1
    int Lc = scol[kHaloW];
    int vc = scol[kHaloW + 1];
    int Rc = scol[kHaloW + 2];
    int hmax_p = max(max(static_cast<int>(scol[0]), static_cast<int>(scol[1])),
                     static_cast<int>(scol[2]));
    unsigned hmin_p = min(min(static_cast<unsigned>(scol[0]),
                              static_cast<unsigned>(scol[1])),
                          static_cast<unsigned>(scol[2]));
    int nlist = 0;
    uint8_t* omax_row = omax + static_cast<int64_t>(g.y0) * out_pitch + g.x0 + lane;
    uint8_t* omin_row = omin + static_cast<int64_t>(g.y0) * out_pitch + g.x0 + lane;
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
        const bool decided =
            col_ok && mx > vc && mn < static_cast<unsigned>(vc);
        if (decided) {
            *omax_row = 0;
            *omin_row = 0;
        }
        omax_row += out_pitch;
        omin_row += out_pitch;
        const bool listed = col_ok && !decided;
        const uint32_t b = __ballot_sync(~0u, listed);
        if (listed) {
            sm.list[nlist + __popc(b & lt_mask)] =
                static_cast<uint16_t>(y * T + lane);
        }
        nlist += __popc(b);
        if (lane == 0) {
            sm.listed[y] = b;
        }
        hmax_p = max(max(Lc, vc), Rc);
        hmin_p = min(min(static_cast<unsigned>(Lc), static_cast<unsigned>(vc)),
                     static_cast<unsigned>(Rc));
        vc = vn;
        Lc = Ln;
        Rc = Rn;
    }
    __syncwarp();

    // -- phase C: flags, seam, dead, links of listed pixels -------------------
    for (int base = 0; base < nlist; base += 32) {
        const int i = base + lane;
        const bool active = i < nlist;
        int p = 0;
        int link0 = -1;
        int link1 = -1;
        if (active) {
            p = sm.list[i];
            const int x = p & 31;
            const int y = p >> 5;
            int nb[9];
            const int16_t* w0 = sm.img + y * kHaloW + x;   // (x-1, y-1)
#pragma unroll
            for (int dy = 0; dy < 3; ++dy) {
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                    nb[dy * 3 + dx] = w0[dy * kHaloW + dx];
                }
            }
            const int v = nb[4];
            const uint32_t rows_up = y > 0 ? sm.listed[y - 1] : 0u;
            const uint32_t rows_c = sm.listed[y];
            const uint32_t rows_dn = y + 1 < g.th ? sm.listed[y + 1] : 0u;
            bool gt = false, lt = false, seam = false, dead = false;
            int parent = p;
            bool have_parent = false;
            // Visit order up, up-left, up-right, left, right, down-left,
            // down, down-right (indices into the 3 x 3 window); the first
            // equal listed predecessor becomes the parent.
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                // k -> window index: 0:U 1:UL 2:UR 3:L 4:R 5:DL 6:D 7:DR
                const int n = k == 0 ? 1 : (k == 1 ? 0 : (k <= 3 ? k : k + 1));
                const int dx = n % 3 - 1;
                const int dy = n / 3 - 1;
                const int nv = nb[n];
                gt |= nv > v;
                lt |= nv >= 0 && nv < v;
                if (nv != v) {
                    continue;
                }
                const int qx = x + dx;
                const int qy = y + dy;
                if (qx < 0 || qx >= T || qy < 0 || qy >= T) {
                    seam = true;
                    continue;
                }
                const uint32_t rowmask =
                    dy < 0 ? rows_up : (dy == 0 ? rows_c : rows_dn);
                if (!((rowmask >> qx) & 1u)) {
                    dead = true;   // an equal decided pixel in the tile
                    continue;
                }
                const bool backward = dy < 0 || (dy == 0 && dx < 0);
                if (!backward) {
                    continue;
                }
                const int q = qy * T + qx;
                if (!have_parent) {
                    parent = q;
                    have_parent = true;
                } else if (n == 2 || n == 3) {
                    // up-right and left edges beyond the chosen parent
                    if (link0 < 0) {
                        link0 = q;
                    } else {
                        link1 = q;
                    }
                }
            }
            const uint32_t own = (gt ? kHasGreater : 0u) |
                                 (lt ? kHasSmaller : 0u) |
                                 (dead ? kDead : 0u) |
                                 (seam ? kTouchesSeam : 0u);
            sm.word[p] = static_cast<uint32_t>(parent) | (own << kOwnShift);
        }
        __syncwarp();
        if (__any_sync(~0u, link0 >= 0)) {
            if (link0 >= 0) wunion(sm.word, p, link0, err);
            if (link1 >= 0) wunion(sm.word, p, link1, err);
        }
        __syncwarp();
    }

    // -- phase D: flatten, zone flags -----------------------------------------
    volatile uint32_t* vw = sm.word;
    for (int base = 0; base < nlist; base += 32) {
        const int i = base + lane;
        if (i < nlist) {
            const int p = sm.list[i];
            int root = p;
#pragma unroll 1
            for (int it = 0; it < T * T; ++it) {
                const int up = static_cast<int>(vw[root] & kParMask);
                if (up == root) break;
                root = up;
            }
            const uint32_t wp = vw[p];
            const uint32_t own = (wp >> kOwnShift) & 7u;
            if (root != p) {
                // p is not a root: no other lane writes its word now.
                vw[p] = (wp & ~kParMask) | static_cast<uint32_t>(root);
            }
            const uint32_t zf = (vw[root] >> kZoneShift) & 7u;
            if ((zf & own) != own) {
                atomicOr(sm.word + root, own << kZoneShift);
            }
        }
    }
    __syncwarp();

    // -- phase E: records, masks of listed pixels, run log --------------------
    // Listed pixels of zones that are final here get their masks now.  Live
    // seam zones are logged as runs (consecutive listed pixels of one row and
    // one zone) and written once, by the resolve pass, with the component's
    // flags.
    const int64_t frag_base = item * kSlots;
    uint32_t* plog = a.pending + item * kPendingCap;
    const uint32_t le_mask = lt_mask | (1u << lane);
    int nrec = 0;
    int nlog = 0;
    for (int base = 0; base < nlist; base += 32) {
        const int i = base + lane;
        const bool active = i < nlist;
        int p = 0;
        int root = 0;
        uint32_t z = 0;
        if (active) {
            p = sm.list[i];
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

    // -- phase F: border records ----------------------------------------------
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
    if (lane < g.tw) {
        border[lane] = static_cast<uint8_t>(record_of(lane, 0));
        border[T + lane] = static_cast<uint8_t>(record_of(lane, g.th - 1));
    }
    if (lane < g.th) {
        border[2 * T + lane] = static_cast<uint8_t>(record_of(0, lane));
        border[3 * T + lane] = static_cast<uint8_t>(record_of(g.tw - 1, lane));
    }
    if (lane == 0) {
        a.fragment_count[item] = static_cast<uint16_t>(min(nrec, kSlots));
        a.pending_count[item] = static_cast<uint32_t>(nlog);
    }

    // -- seam relations --------------------------------------------------------
    // A relation is active when a pixel of this tile equals its 8-neighbour
    // across that seam; both tiles of the pair see the same pixel pairs.
    // Staged pixel (x, y) of the tile, x and y in -1 .. T (rows up to th).
    auto own_px = [&](int x, int y) -> int {
        return sm.img[(y + 1) * kHaloW + x + 1];
    };
    uint32_t rel = 0u;
    {
        const int y = lane;   // left / right columns: lane = row
        if (y < g.th) {
            const int vl = own_px(0, y);
            const int vr = own_px(g.tw - 1, y);
            if (g.x0 > 0) {
                for (int d = -1; d <= 1; ++d) {
                    const int yy = y + d;
                    if (own_px(-1, yy) == vl) {
                        rel |= 1u << (yy < 0 ? kRelTopLeft
                                             : (yy >= T ? kRelBottomLeft
                                                        : kRelLeft));
                    }
                }
            }
            if (g.tw == T && g.x0 + T < width) {
                for (int d = -1; d <= 1; ++d) {
                    const int yy = y + d;
                    if (own_px(T, yy) == vr) {
                        rel |= 1u << (yy < 0 ? kRelTopRight
                                             : (yy >= T ? kRelBottomRight
                                                        : kRelRight));
                    }
                }
            }
        }
        const int x = lane;   // top / bottom rows: lane = column
        if (x < g.tw) {
            const int vt = own_px(x, 0);
            const int vb = own_px(x, g.th - 1);
            if (g.y0 > 0) {
                for (int d = -1; d <= 1; ++d) {
                    const int xx = x + d;
                    if (xx >= 0 && xx < T && own_px(xx, -1) == vt) {
                        rel |= 1u << kRelTop;
                    }
                }
            }
            if (g.th == T && g.y0 + T < height) {
                for (int d = -1; d <= 1; ++d) {
                    const int xx = x + d;
                    if (xx >= 0 && xx < T && own_px(xx, T) == vb) {
                        rel |= 1u << kRelBottom;
                    }
                }
            }
        }
    }
    rel = __reduce_or_sync(~0u, rel);
    uint32_t second = 0u;
    const int64_t tiles_x = job.tiles_x;
    if (rel) {
        __threadfence();
        __syncwarp();
        uint32_t mine = 0u;
        if (lane < 8 && ((rel >> lane) & 1u)) {
            int64_t idx;
            switch (lane) {
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
                mine = 1u << lane;
            }
        }
        second = __reduce_or_sync(~0u, mine);
        if (second) {
            __threadfence();
        }
    }
    // Joins own border pixel (ox, oy) with the outside pixel whose record is
    // byte `off` of tile ng's border records.
    auto join = [&](int ox, int oy, int64_t ng, int off) {
        const uint32_t ro = record_of(ox, oy);
        const uint32_t rn = ld_cg_u8(a.border + ng * kSlots + off);
        const int64_t nbase = ng * kSlots;
        if (ro == kNoRecord || rn == kNoRecord) {
            err = kErrInvariant;   // equal across a seam, yet no seam zone
            return;
        }
        if ((ro != kDeadRecord && ro >= static_cast<uint32_t>(kSlots)) ||
            (rn != kDeadRecord && rn >= static_cast<uint32_t>(kSlots))) {
            err = kErrRecordRange;
            return;
        }
        if (ro == kDeadRecord && rn == kDeadRecord) {
            return;
        }
        if (ro == kDeadRecord) {
            global_or(a.parent, a.bits, static_cast<int>(nbase + rn), kDead,
                      err);
        } else if (rn == kDeadRecord) {
            global_or(a.parent, a.bits, static_cast<int>(frag_base + ro),
                      kDead, err);
        } else {
            global_union(a.parent, a.bits, static_cast<int>(frag_base + ro),
                         static_cast<int>(nbase + rn), err);
        }
    };
    while (second) {
        const int r = __ffs(second) - 1;
        second &= second - 1u;
        if (r == kRelLeft || r == kRelRight) {
            const bool left = r == kRelLeft;
            const int64_t ng = left ? item - 1 : item + 1;
            const int ox = left ? 0 : T - 1;
            const int nx = left ? -1 : T;
            const int side = left ? 3 : 2;   // neighbour's right / left column
            const int y = lane;
            if (y < g.th) {
                const int v = own_px(ox, y);
                for (int d = -1; d <= 1; ++d) {
                    const int y2 = y + d;
                    if (y2 < 0 || y2 >= g.th || own_px(nx, y2) != v) continue;
                    join(ox, y, ng, side * T + y2);
                }
            }
        } else if (r == kRelTop || r == kRelBottom) {
            const bool top = r == kRelTop;
            const int64_t ng = top ? item - tiles_x : item + tiles_x;
            const int oy = top ? 0 : T - 1;
            const int ny = top ? -1 : T;
            const int side = top ? 1 : 0;    // neighbour's bottom / top row
            const int x = lane;
            if (x < g.tw) {
                const int v = own_px(x, oy);
                for (int d = -1; d <= 1; ++d) {
                    const int x2 = x + d;
                    if (x2 < 0 || x2 >= g.tw || own_px(x2, ny) != v) continue;
                    join(x, oy, ng, side * T + x2);
                }
            }
        } else if (lane == 0) {
            int ox, oy, nx, ny, off;
            int64_t ng;
            switch (r) {
                case kRelTopLeft:   // its bottom-right pixel
                    ox = 0; oy = 0; nx = -1; ny = -1; off = T + (T - 1);
                    ng = item - tiles_x - 1; break;
                case kRelTopRight:  // its bottom-left pixel
                    ox = T - 1; oy = 0; nx = T; ny = -1; off = T;
                    ng = item - tiles_x + 1; break;
                case kRelBottomRight:  // its top-left pixel
                    ox = T - 1; oy = T - 1; nx = T; ny = T; off = 0;
                    ng = item + tiles_x + 1; break;
                default:  // bottom-left: its top-right pixel
                    ox = 0; oy = T - 1; nx = -1; ny = T; off = T - 1;
                    ng = item + tiles_x - 1; break;
            }
            const int v = own_px(ox, oy);
            if (v >= 0 && own_px(nx, ny) == v) {
                join(ox, oy, ng, off);
            }
        }
    }
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(item));
    }
}

// ---------------------------------------------------------------------------
// Resolve pass (one warp, one tile)
// ---------------------------------------------------------------------------

struct __align__(16) ResolveSmem {
    uint8_t final_flags[kSlots];
};

__device__ __forceinline__ void resolve_warp(ResolveSmem& sm,
                                             const Source& src,
                                             const Arena& a, int64_t item) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    // The tile pass is complete: clear this tile's seam-pair counters.
    if (lane < 4) {
        a.relation[item * 4 + lane] = 0u;
    }
    const uint32_t n = a.pending_count[item];
    if (n == 0u) {
        return;
    }
    uint32_t err = 0;
    const int count = a.fragment_count[item];
    const int64_t frag_base = item * kSlots;
    uint32_t any = 0u;
#pragma unroll
    for (int i = 0; i < kSlots / 32; ++i) {
        const int r = lane + 32 * i;
        bool flip = false;
        if (r < count) {
            const int f = static_cast<int>(frag_base + r);
            const int root = global_find(a.parent, f, err);
            const uint32_t comp = ld_relaxed(a.bits + root) & 3u;
            const uint32_t own = (ld_relaxed(a.bits + f) >> kLocalShift) & 3u;
            flip = comp != own;
            sm.final_flags[r] = static_cast<uint8_t>(comp);
        }
        any |= __ballot_sync(~0u, flip);
    }
    __syncwarp();
    const PlanImage job = load_job(src, item);
    const TileGeom g = tile_geom(job, item - job.tile_base);
    const int64_t out_pitch = job.out_pitch;
    const uint32_t* plog = a.pending + item * kPendingCap;
    const uint32_t total = min(n, static_cast<uint32_t>(kPendingCap));
    for (uint32_t e = lane; e < total; e += 32) {
        const uint32_t ent = __ldcg(plog + e);
        const int rec = static_cast<int>(ent & 0xFFu);
        const int x = static_cast<int>((ent >> 8) & 63u);
        const int y = static_cast<int>((ent >> 14) & 63u);
        const int len = static_cast<int>((ent >> 20) & 127u);
        if (rec >= count || x + len > g.tw || y >= g.th || len == 0) {
            err = kErrRecordRange;
            continue;
        }
        const uint32_t fl = sm.final_flags[rec];
        const uint8_t mx = (fl & kHasGreater) ? 0 : 255;
        const uint8_t mn = (fl & kHasSmaller) ? 0 : 255;
        const int64_t o = (g.y0 + y) * out_pitch + g.x0 + x;
        for (int k = 0; k < len; ++k) {
            job.maxima[o + k] = mx;
            job.minima[o + k] = mn;
        }
    }
    if (lane == 0 && any) {
        atomicAdd(&a.header->flipped_tiles, 1u);
    }
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(item));
    }
}

}  // namespace rowscan

}  // namespace ss

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
//            both set) get fragment records 0..k-1, the listed pixels'
//            masks are written (provisional for live seam zones), and every
//            pixel of a live seam zone is logged for the resolve pass;
//   phase F  border records: the fragment record of each border pixel, or
//            kDeadRecord when its zone is decided.
//
// Seam merging is wait-free: each pair of tiles joined by equal pixels owns a
// counter and the second tile to arrive unites the pair's live fragments, or
// ORs "both flags" into a live fragment whose partner across the seam is
// dead.  The resolve pass compares every live fragment's own flags with its
// component's and rewrites the logged pixels of the fragments that changed.
#pragma once

#include "ss_device.cuh"

namespace ss {

namespace rowscan {

constexpr int T = 32;
constexpr int kSlots = 4 * T;          // fragment slots per tile
constexpr int kPendingCap = T * T;     // logged pixels per tile
constexpr uint8_t kDeadRecord = 0xFE;  // border record of a decided zone
constexpr uint8_t kNoRecord = 0xFF;    // border pixel of a zone inside the tile

// Per-pixel shared word: bits 0-9 parent, 10-12 zone flags (at roots),
// 13-20 record + 1 (at roots of live seam zones), 21-23 own flags.
constexpr uint32_t kParMask = 0x3FFu;
constexpr int kZoneShift = 10;
constexpr int kRecShift = 13;
constexpr int kOwnShift = 21;
constexpr uint32_t kDead = kHasGreater | kHasSmaller;

struct __align__(16) WarpSmem {
    uint32_t word[T * T];
    uint16_t list[T * T];      // listed (undecided) pixels, in pixel order
    uint32_t listed[T];        // per row: listed pixels
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

__device__ __forceinline__ int wfind(volatile uint32_t* w, int x,
                                     uint32_t& err) {
#pragma unroll 1
    for (int it = 0; it < T * T; ++it) {
        const int p = static_cast<int>(w[x] & kParMask);
        if (p == x) {
            return x;
        }
        x = p;
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

    // -- phase A: flags, decided pixels, list ---------------------------------
    const bool col_ok = lane < g.tw;
    const int gx = g.x0 + lane;
    const bool halo_l = lane == 0 && g.x0 > 0;
    const bool halo_r = lane == 31 && g.x0 + T < width;
    auto load_row = [&](int y, int& v, int& L, int& R) {
        const int gy = g.y0 + y;
        const bool row_ok =
            static_cast<unsigned>(gy) < static_cast<unsigned>(height);
        const uint8_t* rowp = img + gy * pitch;
        v = (row_ok && col_ok) ? static_cast<int>(__ldg(rowp + gx)) : -1;
        int hl = -1;
        int hr = -1;
        if (row_ok && halo_l) hl = static_cast<int>(__ldg(rowp + g.x0 - 1));
        if (row_ok && halo_r) hr = static_cast<int>(__ldg(rowp + g.x0 + T));
        L = __shfl_up_sync(~0u, v, 1);
        R = __shfl_down_sync(~0u, v, 1);
        L = lane == 0 ? hl : L;
        R = lane == 31 ? hr : R;
    };
    int vp, Lp, Rp, vc, Lc, Rc;
    load_row(-1, vp, Lp, Rp);
    load_row(0, vc, Lc, Rc);
    int hmax_p = max(max(Lp, vp), Rp);
    unsigned hmin_p =
        min(min(static_cast<unsigned>(Lp), static_cast<unsigned>(vp)),
            static_cast<unsigned>(Rp));
    int nlist = 0;
#pragma unroll 2
    for (int y = 0; y < g.th; ++y) {
        int vn, Ln, Rn;
        load_row(y + 1, vn, Ln, Rn);
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
            const int64_t o = (g.y0 + y) * out_pitch + gx;
            omax[o] = 0;
            omin[o] = 0;
        }
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
    // Interior tiles (all 8-neighbours inside the image) skip bounds checks.
    const bool interior = g.x0 > 0 && g.y0 > 0 && g.x0 + T < width &&
                          g.y0 + T < height;
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
            const int px = g.x0 + x;
            const int py = g.y0 + y;
            int nb[9];
            if (interior) {
                const uint8_t* r0 = img + (py - 1) * pitch + px - 1;
#pragma unroll
                for (int dy = 0; dy < 3; ++dy) {
#pragma unroll
                    for (int dx = 0; dx < 3; ++dx) {
                        nb[dy * 3 + dx] =
                            static_cast<int>(__ldg(r0 + dy * pitch + dx));
                    }
                }
            } else {
#pragma unroll
                for (int dy = 0; dy < 3; ++dy) {
#pragma unroll
                    for (int dx = 0; dx < 3; ++dx) {
                        nb[dy * 3 + dx] = pixel_at(img, pitch, width, height,
                                                   px + dx - 1, py + dy - 1);
                    }
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

    // -- phase E: records, masks of listed pixels, log ------------------------
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
        if (active) {
            const int x = p & 31;
            const int y = p >> 5;
            const int64_t o = (g.y0 + y) * out_pitch + g.x0 + x;
            omax[o] = (z & kHasGreater) ? 0 : 255;
            omin[o] = (z & kHasSmaller) ? 0 : 255;
        }
        uint32_t rec1 = 0;
        if (live) {
            rec1 = (vw[root] >> kRecShift) & 0xFFu;
        }
        const bool log = live && rec1 != 0u;
        const uint32_t lb = __ballot_sync(~0u, log);
        if (log) {
            plog[nlog + __popc(lb & lt_mask)] =
                static_cast<uint32_t>(p) | ((rec1 - 1u) << 10);
        }
        nlog += __popc(lb);
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
    auto own_px = [&](int x, int y) {
        return pixel_at(img, pitch, width, height, g.x0 + x, g.y0 + y);
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

__device__ __forceinline__ void resolve_warp(WarpSmem& sm, const Source& src,
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
    uint32_t flips[kSlots / 32];
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
        flips[i] = __ballot_sync(~0u, flip);
    }
    uint32_t any = 0u;
#pragma unroll
    for (int i = 0; i < kSlots / 32; ++i) {
        any |= flips[i];
    }
    if (any) {
        __syncwarp();
        const PlanImage job = load_job(src, item);
        const TileGeom g = tile_geom(job, item - job.tile_base);
        const int64_t out_pitch = job.out_pitch;
        const uint32_t* plog = a.pending + item * kPendingCap;
        const uint32_t total = min(n, static_cast<uint32_t>(kPendingCap));
        for (uint32_t e = lane; e < total; e += 32) {
            const uint32_t ent = __ldcg(plog + e);
            const int p = static_cast<int>(ent & 0x3FFu);
            const int rec = static_cast<int>(ent >> 10);
            const int x = p & 31;
            const int y = p >> 5;
            if (rec >= count || x >= g.tw || y >= g.th) {
                err = kErrRecordRange;
                continue;
            }
            uint32_t word = 0u;
#pragma unroll
            for (int i = 0; i < kSlots / 32; ++i) {
                if ((rec >> 5) == i) word = flips[i];
            }
            if (!((word >> (rec & 31)) & 1u)) {
                continue;
            }
            const uint32_t fl = sm.final_flags[rec];
            const int64_t o = (g.y0 + y) * out_pitch + g.x0 + x;
            job.maxima[o] = (fl & kHasGreater) ? 0 : 255;
            job.minima[o] = (fl & kHasSmaller) ? 0 : 255;
        }
        if (lane == 0) {
            atomicAdd(&a.header->flipped_tiles, 1u);
        }
    }
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(item));
    }
}

}  // namespace rowscan

}  // namespace ss

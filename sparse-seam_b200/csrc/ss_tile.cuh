// ss_tile.cuh -- the per-tile labelling worker shared by the tile pass and the
// resolve pass.
//
// A CTA of NW warps owns one T x T tile at a time.  Phases (a __syncthreads
// between each):
//   load       tile + one-pixel halo -> shared memory as int16, -1 = outside
//              the image;
//   predicates per pixel: greater / smaller neighbour, the four backward
//              equal edges inside the tile, equal neighbours outside the tile
//              per seam relation; ballots -> row bitmasks;
//   unions     one union per pair of 8-adjacent equal runs in rows y-1, y;
//   flatten    run heads -> root; OR of the run's flags into the root;
//   number     seam-touching roots get records 0..k-1 in pixel order (a
//              deterministic numbering, so the resolve pass can recompute it).
#pragma once

#include "ss_device.cuh"

namespace ss {

template <int T>
struct __align__(16) TileSmem {
    static constexpr int kHalo = T + 2;
    static constexpr int kChunks = T * T / 32;
    int16_t img[kHalo * kHalo + 4];
    int32_t parent[T * T];
    uint32_t bits[T * T];
    uint32_t m_valid[kChunks];
    uint32_t m_eql[kChunks];
    uint32_t m_gt[kChunks];
    uint32_t m_lt[kChunks];
    uint32_t m_seam[kChunks];
    int32_t chunk_pre[kChunks];
    uint8_t flip[4 * T];
    uint8_t final_flags[4 * T];
    PlanImage job;
    int64_t item;
    int32_t nfrag;
    uint32_t relations;
    uint32_t second;
    int32_t any_flip;
};

template <int T>
__device__ __forceinline__ uint64_t row_mask(const uint32_t* m, int r) {
    if constexpr (T == 32) {
        return m[r];
    } else if constexpr (T == 16) {
        return (m[r >> 1] >> ((r & 1) * 16)) & 0xFFFFu;
    } else {
        return static_cast<uint64_t>(m[2 * r]) |
               (static_cast<uint64_t>(m[2 * r + 1]) << 32);
    }
}

template <int T, int NW>
struct TileWorker {
    static constexpr int kPixels = T * T;
    static constexpr int kHalo = T + 2;
    static constexpr int kChunks = kPixels / 32;
    static constexpr int kPerWarp = kChunks / NW;
    static constexpr int kSlots = 4 * T;
    static constexpr int kLog = T == 16 ? 4 : (T == 32 ? 5 : 6);
    static constexpr int kBound = kPixels + 8;
    static_assert(T == 16 || T == 32 || T == 64, "tile must be 16, 32 or 64");
    static_assert(kChunks % NW == 0, "warps must divide the tile's chunks");

    TileSmem<T>& s;
    const int warp;
    const int lane;
    // Per chunk owned by this lane: bit 0 valid, 1 eq-up, 2 eq-up-left,
    // 3 eq-up-right, 4 seam root (after number()); bits 8-15 run head column.
    uint32_t pred[kPerWarp];
    uint32_t ballot_root[kPerWarp];
    uint32_t err = 0;

    // Tile geometry.
    int x0 = 0, y0 = 0, tw = 0, th = 0, tx = 0, ty = 0;

    __device__ __forceinline__ TileWorker(TileSmem<T>& smem)
        : s(smem),
          warp(static_cast<int>(threadIdx.x) >> 5),
          lane(static_cast<int>(threadIdx.x) & 31) {}

    __device__ __forceinline__ void set_tile(const PlanImage& job,
                                             int64_t local) {
        ty = static_cast<int>(local / job.tiles_x);
        tx = static_cast<int>(local - static_cast<int64_t>(ty) * job.tiles_x);
        x0 = tx * T;
        y0 = ty * T;
        tw = min(T, job.width - x0);
        th = min(T, job.height - y0);
    }

    __device__ __forceinline__ static int chunk_of(int k, int warp_) {
        return warp_ + k * NW;
    }

    // -- load -------------------------------------------------------------
    __device__ __forceinline__ void load(const PlanImage& job) {
        const uint8_t* __restrict__ image = job.image;
        const int width = job.width;
        const int height = job.height;
        const int64_t pitch = job.pitch;
        const int levels = job.levels;
        const bool quantise = levels_active(levels);
        for (int i = static_cast<int>(threadIdx.x); i < kHalo * kHalo;
             i += NW * 32) {
            const int r = i / kHalo;
            const int c = i - r * kHalo;
            const int gy = y0 + r - 1;
            const int gx = x0 + c - 1;
            int v = -1;
            if (static_cast<unsigned>(gy) < static_cast<unsigned>(height) &&
                static_cast<unsigned>(gx) < static_cast<unsigned>(width)) {
                v = __ldg(image + gy * pitch + gx);
                if (quantise) {
                    v = quantize_level(v, levels);
                }
            }
            s.img[i] = static_cast<int16_t>(v);
        }
        if (threadIdx.x == 0) {
            s.relations = 0u;
            s.second = 0u;
        }
    }

    // -- predicates -------------------------------------------------------
    __device__ __forceinline__ void predicates() {
#pragma unroll
        for (int k = 0; k < kPerWarp; ++k) {
            const int c = chunk_of(k, warp);
            const int p = c * 32 + lane;
            const int ly = p >> kLog;
            const int lx = p & (T - 1);
            const int16_t* q = s.img + ly * kHalo + lx;
            const int nUL = q[0], nU = q[1], nUR = q[2];
            const int nL = q[kHalo], v = q[kHalo + 1], nR = q[kHalo + 2];
            const int nDL = q[2 * kHalo], nD = q[2 * kHalo + 1],
                      nDR = q[2 * kHalo + 2];
            const bool valid = v >= 0;
            // Outside pixels are -1: never greater (signed max) and never
            // smaller (unsigned min) than a valid value, never equal to it.
            const int mx = max(max(max(nUL, nU), max(nUR, nL)),
                               max(max(nR, nDL), max(nD, nDR)));
            const unsigned mn =
                min(min(min(static_cast<unsigned>(nUL), static_cast<unsigned>(nU)),
                        min(static_cast<unsigned>(nUR), static_cast<unsigned>(nL))),
                    min(min(static_cast<unsigned>(nR), static_cast<unsigned>(nDL)),
                        min(static_cast<unsigned>(nD), static_cast<unsigned>(nDR))));
            const bool gt = valid && mx > v;
            const bool lt = valid && mn < static_cast<unsigned>(v);
            const bool eL = valid && lx > 0 && nL == v;
            const bool eU = valid && ly > 0 && nU == v;
            const bool eUL = valid && lx > 0 && ly > 0 && nUL == v;
            const bool eUR = valid && ly > 0 && lx < T - 1 && nUR == v;
            uint32_t rel = 0u;
            if (valid) {
                if (ly == 0) {
                    if (nUL == v) rel |= 1u << (lx == 0 ? kRelTopLeft : kRelTop);
                    if (nU == v) rel |= 1u << kRelTop;
                    if (nUR == v) rel |= 1u << (lx == T - 1 ? kRelTopRight : kRelTop);
                }
                if (ly == T - 1) {
                    if (nDL == v) rel |= 1u << (lx == 0 ? kRelBottomLeft : kRelBottom);
                    if (nD == v) rel |= 1u << kRelBottom;
                    if (nDR == v) rel |= 1u << (lx == T - 1 ? kRelBottomRight : kRelBottom);
                }
                if (lx == 0) {
                    if (ly > 0 && nUL == v) rel |= 1u << kRelLeft;
                    if (nL == v) rel |= 1u << kRelLeft;
                    if (ly < T - 1 && nDL == v) rel |= 1u << kRelLeft;
                }
                if (lx == T - 1) {
                    if (ly > 0 && nUR == v) rel |= 1u << kRelRight;
                    if (nR == v) rel |= 1u << kRelRight;
                    if (ly < T - 1 && nDR == v) rel |= 1u << kRelRight;
                }
            }
            const uint32_t b_valid = __ballot_sync(~0u, valid);
            const uint32_t b_eql = __ballot_sync(~0u, eL);
            const uint32_t b_gt = __ballot_sync(~0u, gt);
            const uint32_t b_lt = __ballot_sync(~0u, lt);
            const uint32_t b_seam = __ballot_sync(~0u, rel != 0u);
            const uint32_t rel_all = __reduce_or_sync(~0u, rel);
            if (lane == 0) {
                s.m_valid[c] = b_valid;
                s.m_eql[c] = b_eql;
                s.m_gt[c] = b_gt;
                s.m_lt[c] = b_lt;
                s.m_seam[c] = b_seam;
                if (rel_all) {
                    atomicOr(&s.relations, rel_all);
                }
            }
            pred[k] = (valid ? 1u : 0u) | (eU ? 2u : 0u) | (eUL ? 4u : 0u) |
                      (eUR ? 8u : 0u);
            s.parent[p] = p;
            s.bits[p] = 0u;
        }
    }

    // Run head (first column of the run) of column x in row r.
    __device__ __forceinline__ int run_head(int r, int x) const {
        const uint64_t heads =
            row_mask<T>(s.m_valid, r) & ~row_mask<T>(s.m_eql, r);
        return high_bit(heads & bits_upto(x));
    }

    // -- unions -----------------------------------------------------------
    // Run R in row y (value v) is 8-adjacent to every run of row y-1 that
    // has a pixel equal to v in columns [head-1, end+1].  Those above-pixels
    // form maximal segments, one per distinct above-run, and each segment's
    // first column is hit by exactly one of:
    //   (a) a pixel x of R with eq-up and not eq-up-left      (segment at x)
    //   (b) the head of R with eq-up-left                    (at head - 1)
    //   (c) the end of R with eq-up-right and not eq-up      (at end + 1)
    __device__ __forceinline__ void unions() {
#pragma unroll
        for (int k = 0; k < kPerWarp; ++k) {
            const int c = chunk_of(k, warp);
            const int p = c * 32 + lane;
            const int ly = p >> kLog;
            const int lx = p & (T - 1);
            const uint32_t pr = pred[k];
            if (!(pr & 1u)) {
                continue;
            }
            const uint64_t eql = row_mask<T>(s.m_eql, ly);
            const uint64_t heads = row_mask<T>(s.m_valid, ly) & ~eql;
            const int head = high_bit(heads & bits_upto(lx));
            pred[k] = pr | (static_cast<uint32_t>(head) << 8);
            if (!(pr & 14u)) {
                continue;
            }
            const bool eU = pr & 2u;
            const bool eUL = pr & 4u;
            const bool eUR = pr & 8u;
            const int me = ly * T + head;
            const uint64_t heads_above =
                row_mask<T>(s.m_valid, ly - 1) & ~row_mask<T>(s.m_eql, ly - 1);
            const int base = (ly - 1) * T;
            if (eU && !eUL) {
                smem_union<kBound>(s.parent, me,
                                   base + high_bit(heads_above & bits_upto(lx)),
                                   err);
            }
            if (lx == head && eUL) {
                smem_union<kBound>(
                    s.parent, me,
                    base + high_bit(heads_above & bits_upto(lx - 1)), err);
            }
            const bool is_end = lx == T - 1 || !((eql >> (lx + 1)) & 1ull);
            if (is_end && eUR && !eU) {
                smem_union<kBound>(
                    s.parent, me,
                    base + high_bit(heads_above & bits_upto(lx + 1)), err);
            }
        }
    }

    // -- flatten ------------------------------------------------------------
    // Read-only finds (other threads store roots concurrently, which only
    // shortens the paths), then each run head stores its root and ORs the
    // run's flags into it.
    __device__ __forceinline__ void flatten() {
#pragma unroll
        for (int k = 0; k < kPerWarp; ++k) {
            const int c = chunk_of(k, warp);
            const int p = c * 32 + lane;
            const int ly = p >> kLog;
            const int lx = p & (T - 1);
            const uint32_t pr = pred[k];
            if (!(pr & 1u) || static_cast<int>((pr >> 8) & 0xFFu) != lx) {
                continue;
            }
            volatile int32_t* par = s.parent;
            int root = p;
#pragma unroll 1
            for (int it = 0; it < kBound; ++it) {
                const int up = par[root];
                if (up == root) {
                    break;
                }
                root = up;
            }
            par[p] = root;
            const uint64_t heads =
                row_mask<T>(s.m_valid, ly) & ~row_mask<T>(s.m_eql, ly);
            const uint64_t later = heads & ~bits_upto(lx);
            const int last = later ? (__ffsll(static_cast<long long>(later)) - 2)
                                   : (T - 1);
            const uint64_t run = bits_upto(last) & ~(bits_upto(lx) >> 1);
            uint32_t f = 0u;
            f |= (row_mask<T>(s.m_gt, ly) & run) ? kHasGreater : 0u;
            f |= (row_mask<T>(s.m_lt, ly) & run) ? kHasSmaller : 0u;
            f |= (row_mask<T>(s.m_seam, ly) & run) ? kTouchesSeam : 0u;
            if (f) {
                atomicOr(&s.bits[root], f);
            }
        }
    }

    // -- number -------------------------------------------------------------
    // Seam roots in pixel order get records 0..k-1.  When `arena` is set, the
    // records' union-find slots are initialised (parent = self, flags = own).
    // Ends with a __syncthreads.
    __device__ __forceinline__ void number(const Arena* arena,
                                           int64_t frag_base) {
#pragma unroll
        for (int k = 0; k < kPerWarp; ++k) {
            const int c = chunk_of(k, warp);
            const int p = c * 32 + lane;
            const int lx = p & (T - 1);
            const uint32_t pr = pred[k];
            const bool root = (pr & 1u) &&
                              static_cast<int>((pr >> 8) & 0xFFu) == lx &&
                              s.parent[p] == p &&
                              (s.bits[p] & kTouchesSeam);
            const uint32_t b = __ballot_sync(~0u, root);
            ballot_root[k] = b;
            if (root) {
                pred[k] = pr | 16u;
            }
            if (lane == 0) {
                s.chunk_pre[c] = __popc(b);
            }
        }
        __syncthreads();
        if (warp == 0) {
            constexpr int kPer = (kChunks + 31) / 32;
            int vals[kPer];
            int sum = 0;
#pragma unroll
            for (int j = 0; j < kPer; ++j) {
                const int idx = lane * kPer + j;
                vals[j] = idx < kChunks ? s.chunk_pre[idx] : 0;
                sum += vals[j];
            }
            int incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int n = __shfl_up_sync(~0u, incl, o);
                if (lane >= o) {
                    incl += n;
                }
            }
            int excl = incl - sum;
#pragma unroll
            for (int j = 0; j < kPer; ++j) {
                const int idx = lane * kPer + j;
                if (idx < kChunks) {
                    s.chunk_pre[idx] = excl;
                }
                excl += vals[j];
            }
            if (lane == 31) {
                s.nfrag = incl;
            }
        }
        __syncthreads();
        const uint32_t below = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < kPerWarp; ++k) {
            if (!(pred[k] & 16u)) {
                continue;
            }
            const int c = chunk_of(k, warp);
            const int p = c * 32 + lane;
            const int rec = s.chunk_pre[c] + __popc(ballot_root[k] & below);
            // A tile has at most 4T - 4 border pixels, hence at most 4T - 4
            // seam zones; the check guards the arena against a broken tile.
            if (rec >= kSlots) {
                err = kErrFragmentOverflow;
                continue;
            }
            const uint32_t f = s.bits[p];
            s.bits[p] = f | (static_cast<uint32_t>(rec + 1) << kRecordShift);
            if (arena) {
                const int64_t g = frag_base + rec;
                arena->parent[g] = static_cast<int32_t>(g);
                arena->bits[g] = (f & 3u) | ((f & 3u) << kLocalShift);
            }
        }
        __syncthreads();
    }

    // Root flags word of pixel (lx, ly): zone flags, TOUCHES_SEAM and, for
    // seam zones, (record + 1) << 8.
    __device__ __forceinline__ uint32_t zone_word(int lx, int ly) const {
        const int head = run_head(ly, lx);
        return s.bits[s.parent[ly * T + head]];
    }
};

}  // namespace ss

// ss_runs.cuh -- the T = 32 tile pass: one warp per 32 x 32 tile, on
// per-row bit masks and runs.
//
// The tile and its one-pixel halo are staged in shared memory, rows t and
// t + 16 paired in one word as two half-precision numbers (NaN outside the
// image).  A row scan (lane = column, two rows per step) finds each pixel's
// greater / smaller flags from sliding 3 x 3 pair maxima / minima (both pass
// over NaN); "decided" pixels have both and are in neither mask, with their
// whole zone.  The scan leaves seven 32-bit masks
// per tile row in the registers of lane y = row:
//   L    listed pixels (not decided)
//   GT   listed pixels with a strictly greater 8-neighbour
//   LT   listed pixels with a strictly smaller 8-neighbour
//   EU   pixels equal to the pixel above          (bit x: v(x,y) == v(x,y-1))
//   EUL  pixels equal to the pixel above-left     (v(x,y) == v(x-1,y-1))
//   EUR  pixels equal to the pixel above-right    (v(x,y) == v(x+1,y-1))
//   EL   pixels equal to the pixel on the left    (v(x,y) == v(x-1,y))
// From these, with shifts and the neighbouring rows' masks (shuffles):
//   runs      maximal horizontal runs of equal listed pixels (heads, ends);
//   dead      listed pixels with an equal decided neighbour in the tile
//             (their zone holds a decided pixel, so it is in no mask);
//   seam      listed pixels with an equal neighbour outside the tile;
//   links     one union per pair of 8-adjacent equal runs in consecutive
//             rows, at the first column of their contact: (a) a pixel equal
//             to the one above and not to the one above-left, (b) a run head
//             equal to the pixel above-left, (c) a run end equal to the pixel
//             above-right and not to the one above.
// Union-find runs over run heads only, one lane per row, so its cost grows
// with the number of runs and contacts per row rather than with the number
// of listed pixels: a large plateau is a few runs per row.  Runs that no
// union touches and no seam reaches are zones of their own: their verdicts
// come from per-run carry tests on the row masks, and the loops over runs
// visit only the others.  Zone flags are
// ORed into the roots; live seam zones (touching a seam, flags not both set)
// get records (numbered as the verdict loop first meets them) and a log of
// their runs; every
// pixel of the tile gets its mask bytes in one final pass, whole rows with
// vector stores where the output allows (live pixels get a placeholder that
// the resolve pass replaces); border records and seam items go to the
// workspace for the seam pass.
//
// Reference behaviour followed (paths inside the reference repository):
// zone flags and seam test, harness/primary/snapshot_sparse_seam_cuda_v1_0.cu
// :340-390; per-tile fragment records, :392-410; cross-seam merge of equal
// 8-adjacent border pixels, :508-581; masks from the resolved flags, :477-506.
#pragma once

#include "ss_rowscan.cuh"

namespace ss {

namespace rowscan {

// The staged square pairs row r with row r + 16 in one 32-bit word: slot s
// (0 .. 17) of staged column c holds staged row s in its low half and staged
// row s + 16 in its high half, so one row-scan step handles tile rows t and
// t + 16 with half-precision pair max / min.  A pixel value v is staged as
// the half 1024 + v (bits 0x6400 | v: exact, ordered, equal iff the values
// are), a pixel outside the image as 0xFFFF, a NaN, which max and min pass
// over.  Staged rows 16 and 17 sit in both halves (low of slots 16, 17;
// high of 0, 1).
constexpr int kSlotRows = T / 2 + 2;
constexpr uint32_t kStageBias = 0x6400u;   // half-precision 1024

__device__ __forceinline__ int16_t stage_code(int v) {
    return static_cast<int16_t>(v >= 0 ? static_cast<int>(kStageBias) | v
                                       : -1);
}

// Per warp (one 32 x 32 square): the seam equality masks kept for the end
// of the pass, and the staged square (its image pixels + halo; slot s of
// staged column c at word 1 + s * kHaloW + c, so that tile columns 4k and
// 4k + 1 share an 8-byte boundary), later reused for the run list.
struct __align__(16) RunAux {
    uint32_t eq[16];
    uint32_t img[kSlotRows * kHaloW + 2];
};
static_assert(sizeof(uint32_t) * (kSlotRows * kHaloW + 2) >=
                  sizeof(uint16_t) * kListCap + sizeof(uint32_t) * 3 * T,
              "the run list and its row masks reuse the staged square");

// Pair maximum / minimum of two staged words, both halves at once; a NaN
// half (outside the image) yields the other operand's half, and a number
// comes back bit for bit.
__device__ __forceinline__ uint32_t max_pair(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("max.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t min_pair(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("min.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// Warp ballots of a pair comparison: bit `lane` of lo / hi is the comparison
// of the lanes' low / high halves (one compare for both, false where either
// half is a NaN).  Every lane of the warp must call it.
#define SS_PAIR_BALLOT(NAME, CMP)                                            \
    __device__ __forceinline__ void NAME(uint32_t a, uint32_t b,            \
                                         uint32_t& lo, uint32_t& hi) {      \
        asm volatile(                                                       \
            "{\n\t.reg .pred p, q;\n\t"                                     \
            "setp." CMP ".f16x2 p|q, %2, %3;\n\t"                           \
            "vote.sync.ballot.b32 %0, p, 0xffffffff;\n\t"                   \
            "vote.sync.ballot.b32 %1, q, 0xffffffff;\n\t}"                  \
            : "=r"(lo), "=r"(hi)                                            \
            : "r"(a), "r"(b));                                              \
    }
SS_PAIR_BALLOT(ballot_pair_gt, "gt")
SS_PAIR_BALLOT(ballot_pair_lt, "lt")
SS_PAIR_BALLOT(ballot_pair_eq, "eq")
#undef SS_PAIR_BALLOT

// Tile edge 32: one warp per tile, its own words.
struct __align__(16) RunSmem {
    uint32_t word[T * T];          // union-find word at each run head
    RunAux aux;
};

// Tile edge 64: four warps per tile, one per 32 x 32 quadrant (q = 2 qy +
// qx), sharing one union-find over the quadrants' run heads (quadrant q's
// words at q * 1024 + ...), and the tile's counters.
struct __align__(16) RunCta {
    uint32_t lmask[4][T];          // listed pixels per quadrant row
    uint32_t hmask[4][T];          // run heads per quadrant row
    uint32_t nrec, nlog, nitems, logged_px;
};

struct __align__(16) RunSmem64 {
    uint32_t word[4 * T * T];
    RunAux aux[4];
    RunCta cta;
};

// Run-head words store the parent as (parent XOR self) in bits 0-9, so an
// all-zero word is a root with no flags: the words start zeroed.
__device__ __forceinline__ int rparent(uint32_t w, int x) {
    return static_cast<int>((w & kParMask) ^ static_cast<uint32_t>(x));
}

__device__ __forceinline__ uint32_t with_parent(uint32_t w, int x, int p) {
    return (w & ~kParMask) | static_cast<uint32_t>(p ^ x);
}

// Find with path halving (used while linking: a non-root word changes only
// in its parent bits, and halving writes an ancestor).  Walks are bounded by
// the number of words of a tile.
constexpr int kWalkBound = 4 * T * T;

__device__ __forceinline__ int rfind(volatile uint32_t* w, int x,
                                     uint32_t& err) {
#pragma unroll 1
    for (int it = 0; it < kWalkBound; ++it) {
        const uint32_t wx = w[x];
        const int p = rparent(wx, x);
        if (p == x) {
            return x;
        }
        const int gp = rparent(w[p], p);
        if (gp == p) {
            return p;
        }
        w[x] = with_parent(wx, x, gp);
        x = gp;
    }
    err = kErrSpinLimit;
    return x;
}

// Links the larger root below the smaller one (CAS on the whole word).
__device__ __forceinline__ void runion(uint32_t* w_, int a, int b,
                                       uint32_t& err) {
    volatile uint32_t* w = w_;
#pragma unroll 1
    for (int it = 0; it < 4 * kWalkBound; ++it) {
        a = rfind(w, a, err);
        b = rfind(w, b, err);
        if (a == b || err) {
            return;
        }
        const int hi = a > b ? a : b;
        const int lo = a > b ? b : a;
        const uint32_t cur = w[hi];
        if (rparent(cur, hi) != hi) {
            continue;
        }
        if (atomicCAS(w_ + hi, cur, with_parent(cur, hi, lo)) == cur) {
            return;
        }
    }
    err = kErrSpinLimit;
}

// Word of the run whose head is column h of row y.  The column is XORed with
// the row so that the lanes of a lane-per-row step, which often touch heads
// in the same column, hit 32 different shared-memory banks; within a row
// the map is a permutation, so every (y, h) keeps its own word.
__device__ __forceinline__ int run_word(int y, int h) {
    return (y << 5) | (h ^ y);
}

// Head of the run holding bit x of a row whose run heads are `heads`.
__device__ __forceinline__ int head_of(uint32_t heads, int x) {
    return 31 - __clz(heads & le_mask_of(x));
}

// Per-run tests by carry propagation.  With `q` marking the pixels whose
// right neighbour continues their run, adding a run's head bit to q sends a
// carry through the run's pixels that stops at its end: (q + H) ^ q is the
// whole of every run whose head is in H.  Started on q & ~m instead, the
// carry stops at the run's first bit of m, and so reaches the run's end
// only when no earlier pixel of the run is in m.
struct RunShape {
    uint32_t q;        // pixels whose right neighbour continues their run
    uint32_t rq;       // the same in bit-reversed order (ends become heads)
    uint32_t rheads;   // run ends, bit-reversed
    uint32_t rends;    // run heads, bit-reversed
};

__device__ __forceinline__ RunShape run_shape(uint32_t cont, uint32_t heads,
                                              uint32_t ends) {
    RunShape s;
    s.q = cont >> 1;
    s.rq = __brev(cont);
    s.rheads = __brev(ends);
    s.rends = __brev(heads);
    return s;
}

// Heads of the runs that hold no bit of m (the carry runs from each run's
// end towards its head in bit-reversed order).
__device__ __forceinline__ uint32_t clean_heads(const RunShape& s,
                                                uint32_t m) {
    const uint32_t rm = __brev(m);
    return __brev(s.rends & ((s.rq & ~rm) + s.rheads) & ~rm);
}

// Every pixel of the runs whose heads are in hs.
__device__ __forceinline__ uint32_t run_span(const RunShape& s, uint32_t hs) {
    return (s.q + hs) ^ s.q;
}

// Bytes 0x00 / 0xFF of the 4 bits of `nib` that sit at bit `shift` of it
// (the other bits of `nib` are masked off): the product places bit i of the
// nibble at bit 7 of byte i (copies shifted by 7, 14, 21 and 28 bits do not
// overlap), and a byte permute that replicates each byte's top bit fills it.
template <int kShift>
__device__ __forceinline__ uint32_t expand4(uint32_t nib) {
    const uint32_t t = (nib & (15u << kShift)) * (0x10204080u >> kShift);
    uint32_t d;
    asm("prmt.b32 %0, %1, 0, 0xBA98;" : "=r"(d) : "r"(t));
    return d;
}

// Writes the 32 x 32 mask bytes of a full tile from per-row bit masks held
// by lane = row (`mxb`, `mnb`: 1 = byte 255), VEC bytes per store (16, 8 or
// 4; rows and bases aligned to it).  Each store instruction covers
// 32 * VEC bytes: 32 / VEC lanes per row, VEC rows per instruction.
template <int VEC>
__device__ __forceinline__ void store_rows(uint8_t* omax, uint8_t* omin,
                                           const TileGeom& g,
                                           int64_t out_pitch, uint32_t mxb,
                                           uint32_t mnb) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    constexpr int kPerRow = T / VEC;
    const int c = lane % kPerRow;
    const int rr = lane / kPerRow;
    const int64_t o =
        static_cast<int64_t>(g.y0 + rr) * out_pitch + g.x0 + c * VEC;
    uint8_t* px = omax + o;
    uint8_t* pn = omin + o;
    const int64_t step = static_cast<int64_t>(VEC) * out_pitch;
#pragma unroll
    for (int r0 = 0; r0 < T; r0 += VEC) {
        const uint32_t bx = __shfl_sync(~0u, mxb, r0 + rr) >> (c * VEC);
        const uint32_t bn = __shfl_sync(~0u, mnb, r0 + rr) >> (c * VEC);
        if constexpr (VEC == 16) {
            *reinterpret_cast<uint4*>(px) =
                make_uint4(expand4<0>(bx), expand4<4>(bx), expand4<0>(bx >> 8),
                           expand4<4>(bx >> 8));
            *reinterpret_cast<uint4*>(pn) =
                make_uint4(expand4<0>(bn), expand4<4>(bn), expand4<0>(bn >> 8),
                           expand4<4>(bn >> 8));
        } else if constexpr (VEC == 8) {
            *reinterpret_cast<uint2*>(px) =
                make_uint2(expand4<0>(bx), expand4<4>(bx));
            *reinterpret_cast<uint2*>(pn) =
                make_uint2(expand4<0>(bn), expand4<4>(bn));
        } else {
            *reinterpret_cast<uint32_t*>(px) = expand4<0>(bx);
            *reinterpret_cast<uint32_t*>(pn) = expand4<0>(bn);
        }
        px += step;
        pn += step;
    }
}

// The tile pass over one tile.  Q = 1: tile edge 32, the calling warp
// labels the whole tile, `words` are its own 1024 union-find words and `cta`
// is unused.  Q = 4: tile edge 64, the calling warp (q = 2 qy + qx) labels
// quadrant q of the tile, `words` are the CTA's 4096 words; every warp of
// the CTA calls this with the same item (it holds __syncthreads).  The
// quadrants' zones are joined in the shared union-find across the inner
// sides, so fragments, records, border records, seam items and the run log
// belong to the 64 x 64 tile.
template <int Q>
__device__ __forceinline__ void tile_pass_runs(uint32_t* words, RunAux& ax,
                                               RunCta* cta, int q,
                                               const Source& src,
                                               const Arena& a,
                                               int64_t item) {
    constexpr int TT = Q == 4 ? 2 * T : T;
    constexpr int kSlotsT = Edge<TT>::kSlots;
    constexpr int kPendingT = Edge<TT>::kPendingCap;
    constexpr int kSeamT = Edge<TT>::kSeamCap;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t err = 0;
    const int wb = q * T * T;          // this warp's first word
    uint32_t* const W = words + wb;
    const int qx = q & 1;
    const int qy = q >> 1;

    const PlanImage job = load_job(src, item);
    const TileGeom tg = tile_geom<TT>(job, item - job.tile_base);
    // This warp's square: the tile, or its quadrant (possibly empty).
    TileGeom g = tg;
    if constexpr (Q == 4) {
        g.x0 = tg.x0 + T * qx;
        g.y0 = tg.y0 + T * qy;
        g.tw = max(0, min(T, tg.tw - T * qx));
        g.th = max(0, min(T, tg.th - T * qy));
        if (threadIdx.x == 0) {
            cta->nrec = 0u;
            cta->nlog = 0u;
            cta->nitems = 0u;
            cta->logged_px = 0u;
        }
    }
    const bool two_cols = Q == 4 && tg.tw > T;
    const bool two_rows = Q == 4 && tg.th > T;
    // Which sides of the square are sides of the tile (the others face
    // another quadrant).
    const bool ext_t = Q == 1 || qy == 0;
    const bool ext_b = Q == 1 || qy == 1 || !two_rows;
    const bool ext_l = Q == 1 || qx == 0;
    const bool ext_r = Q == 1 || qx == 1 || !two_cols;
    const uint8_t* __restrict__ img = job.image;
    const int64_t pitch = job.pitch;
    const int width = job.width;
    const int height = job.height;
    const int64_t out_pitch = job.out_pitch;
    uint8_t* __restrict__ omax = job.maxima;
    uint8_t* __restrict__ omin = job.minima;
    uint32_t* const simg = ax.img + 1;
    int16_t* const shalf = reinterpret_cast<int16_t*>(simg);

    // -- prologue: stage the tile and its halo; zero the words --------------
    // Staged row r holds image row y0 - 1 + r, staged column c image column
    // x0 - 1 + c; slot s of column c (word s * kHaloW + c of simg) pairs
    // staged rows s and s + 16.
    {
        // Optional re-quantisation of every loaded pixel through a 256-entry
        // table in the (not yet used) union-find words, built before the
        // loads so that it does not hold registers while they are in flight.
        const bool quantise = levels_active(job.levels);
        const uint8_t* lut = reinterpret_cast<const uint8_t*>(W);
        if (quantise) {
            uint8_t* t8 = reinterpret_cast<uint8_t*>(W);
#pragma unroll 1
            for (int k = 0; k < 8; ++k) {
                const int v = k * 32 + lane;
                t8[v] = static_cast<uint8_t>(quantize_level(v, job.levels));
            }
            __syncwarp();
        }
        // Halo columns x0 - 1 and x0 + T of staged rows 0..33 (lanes 0..31,
        // then lanes 0..1 for rows 32..33).
        const int xl = g.x0 - 1;
        const int xr = g.x0 + T;
        const int gy0 = g.y0 - 1 + lane;
        const int gy1 = g.y0 + 31 + lane;
        // (An empty quadrant, beyond the image, loads nothing.)
        const bool any = g.tw > 0 && g.th > 0;
        const bool ok0 = any &&
            static_cast<unsigned>(gy0) < static_cast<unsigned>(height);
        const bool ok1 = any && lane < 2 && static_cast<unsigned>(gy1) <
                                         static_cast<unsigned>(height);
        auto load_halo = [&](int& hl0, int& hr0, int& hl1, int& hr1) {
            hl0 = (xl >= 0 && ok0)
                      ? static_cast<int>(__ldg(img + gy0 * pitch + xl))
                      : -1;
            hr0 = (xr < width && ok0)
                      ? static_cast<int>(__ldg(img + gy0 * pitch + xr))
                      : -1;
            hl1 = (xl >= 0 && ok1)
                      ? static_cast<int>(__ldg(img + gy1 * pitch + xl))
                      : -1;
            hr1 = (xr < width && ok1)
                      ? static_cast<int>(__ldg(img + gy1 * pitch + xr))
                      : -1;
        };
        // Staged row r, column c, into its half-word(s).
        auto put = [&](int r, int c, int16_t v) {
            if (r < kSlotRows) {
                shalf[2 * (r * kHaloW + c)] = v;
            }
            if (r >= T / 2) {
                shalf[2 * ((r - T / 2) * kHaloW + c) + 1] = v;
            }
        };
        auto store_halo = [&](int16_t hl0, int16_t hr0, int16_t hl1,
                              int16_t hr1) {
            put(lane, 0, hl0);
            put(lane, kHaloW - 1, hr0);
            if (lane < 2) {
                put(32 + lane, 0, hl1);
                put(32 + lane, kHaloW - 1, hr1);
            }
        };
        int hl0, hr0, hl1, hr1;
        // A tile whose halo lies inside the image, in an image whose rows
        // start on 4-byte boundaries, is read 4 pixels per lane: 8 lanes per
        // row, 4 rows per load instruction.  Lane (k, rr) holds staged rows
        // rr + 4i, so rows s and s + 16 of its slots s = rr + 4j are its
        // words j and j + 4, which widen into the slot's 4 packed words.
        const bool word_rows =
            g.tw > 0 && g.th > 0 &&
            !quantise && g.x0 > 0 && g.y0 > 0 && g.x0 + T < width &&
            g.y0 + T < height &&
            ((reinterpret_cast<uintptr_t>(img) |
              static_cast<uintptr_t>(pitch)) & 3u) == 0;
        if (word_rows) {
            const int k = lane & 7;
            const int rr = lane >> 3;
            const uint8_t* src =
                img + static_cast<int64_t>(g.y0 - 1 + rr) * pitch + g.x0 + 4 * k;
            uint2* dst = reinterpret_cast<uint2*>(simg + rr * kHaloW + 1 + 4 * k);
            uint32_t w[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                w[i] = (i < 8 || rr < 2)
                           ? __ldg(reinterpret_cast<const uint32_t*>(
                                 src + static_cast<int64_t>(4 * i) * pitch))
                           : 0u;
            }
            load_halo(hl0, hr0, hl1, hr1);
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                if (j < 4 || rr < 2) {
                    // Bytes m of the rows s and s + 16 -> (row s) | (row
                    // s + 16) << 16 for the slot's columns 4k + m.
                    const uint32_t t01 = __byte_perm(w[j], w[j + 4], 0x5140);
                    const uint32_t t23 = __byte_perm(w[j], w[j + 4], 0x7362);
                    uint2* d = dst + j * 2 * kHaloW;
                    // Byte 4 of the selector is the bias's high byte.
                    const uint32_t hb = kStageBias >> 8;
                    d[0] = make_uint2(__byte_perm(t01, hb, 0x4140),
                                      __byte_perm(t01, hb, 0x4342));
                    d[1] = make_uint2(__byte_perm(t23, hb, 0x4140),
                                      __byte_perm(t23, hb, 0x4342));
                }
            }
            store_halo(stage_code(hl0), stage_code(hr0), stage_code(hl1),
                       stage_code(hr1));
        } else {
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
            load_halo(hl0, hr0, hl1, hr1);
            if (quantise) {
                auto q = [&](int v) -> int16_t {
                    return stage_code(v >= 0 ? lut[v] : v);
                };
#pragma unroll
                for (int r = 0; r < kSlotRows; ++r) {
                    simg[r * kHaloW + lane + 1] =
                        static_cast<uint16_t>(q(vals[r])) |
                        static_cast<uint32_t>(
                            static_cast<uint16_t>(q(vals[r + T / 2]))) << 16;
                }
                store_halo(q(hl0), q(hr0), q(hl1), q(hr1));
            } else {
#pragma unroll
                for (int r = 0; r < kSlotRows; ++r) {
                    simg[r * kHaloW + lane + 1] =
                        static_cast<uint16_t>(stage_code(vals[r])) |
                        static_cast<uint32_t>(static_cast<uint16_t>(
                            stage_code(vals[r + T / 2]))) << 16;
                }
                store_halo(stage_code(hl0), stage_code(hr0), stage_code(hl1),
                           stage_code(hr1));
            }
        }
        __syncwarp();
        // Words 0..255 first carry the row masks of the scan and are
        // cleared after it.
        uint4* w4 = reinterpret_cast<uint4*>(W);
#pragma unroll
        for (int k = 2; k < T * T / 128; ++k) {
            w4[k * 32 + lane] = make_uint4(0u, 0u, 0u, 0u);
        }
    }
    __syncwarp();

    // -- row scan: flags, decided pixels, row masks ----------------------------
    const bool col_ok = lane < g.tw;
    uint32_t rL = 0, rGT = 0, rLT = 0, rEU = 0, rEUL = 0, rEUR = 0, rEL = 0;
    // Bottom seam of a full-height tile: bit x of bEq[d + 1] is pixel
    // (x, T - 1) equal to pixel (x + d, T) below the tile (d = -1, 0, 1).
    uint32_t bEq[3] = {0u, 0u, 0u};
    {
        // Step t handles tile rows t (low halves) and t + 16 (high halves):
        // slots t, t + 1, t + 2 hold staged rows t .. t + 2 and t + 16 ..
        // t + 18.  Rows at or beyond the tile's height give masks that the
        // pick-up below ignores.
        const uint32_t* scol = simg + lane;   // staged columns lane .. lane + 2
        uint32_t Lp = scol[0];
        uint32_t vp = scol[1];
        uint32_t Rp = scol[2];
        uint32_t Lc = scol[kHaloW];
        uint32_t vc = scol[kHaloW + 1];
        uint32_t Rc = scol[kHaloW + 2];
        uint32_t hmax_p = max_pair(max_pair(Lp, vp), Rp);
        uint32_t hmin_p = min_pair(min_pair(Lp, vp), Rp);
        uint32_t hmax_c = max_pair(max_pair(Lc, vc), Rc);
        uint32_t hmin_c = min_pair(min_pair(Lc, vc), Rc);
        const int steps = min(g.th, T / 2);
#pragma unroll 2
        for (int t = 0; t < steps; ++t) {
            const uint32_t* nrow = scol + (t + 2) * kHaloW;
            const uint32_t Ln = nrow[0];
            const uint32_t vn = nrow[1];
            const uint32_t Rn = nrow[2];
            const uint32_t hmax_n = max_pair(max_pair(Ln, vn), Rn);
            const uint32_t hmin_n = min_pair(min_pair(Ln, vn), Rn);
            // 3 x 3 maxima / minima including the centre: a neighbour is
            // greater iff the maximum of the nine is above the centre,
            // smaller iff the minimum is below it.
            const uint32_t mx = max_pair(max_pair(hmax_p, hmax_c), hmax_n);
            const uint32_t mn = min_pair(min_pair(hmin_p, hmin_c), hmin_n);
            // Lane y derives its row's listed / greater / smaller masks from
            // these after the scan.  A pixel outside the image (NaN) is
            // equal to none; every use of the equality masks is restricted
            // to listed pixels, which are inside.
            uint32_t bG0, bG1, bS0, bS1, bEU0, bEU1, bEUL0, bEUL1, bEUR0,
                bEUR1, bEL0, bEL1;
            ballot_pair_gt(mx, vc, bG0, bG1);
            ballot_pair_lt(mn, vc, bS0, bS1);
            ballot_pair_eq(vc, vp, bEU0, bEU1);
            ballot_pair_eq(vc, Lp, bEUL0, bEUL1);
            ballot_pair_eq(vc, Rp, bEUR0, bEUR1);
            ballot_pair_eq(vc, Lc, bEL0, bEL1);
            if (lane == 0) {
                // Rows t and t + 16's masks, picked up by lanes t and t + 16
                // after the scan.
                uint4* slot = reinterpret_cast<uint4*>(W + 8 * t);
                slot[0] = make_uint4(bG0, bS0, bEU0, bEUL0);
                slot[1] = make_uint4(bEUR0, bEL0, 0u, 0u);
                uint4* slot1 = reinterpret_cast<uint4*>(W + 8 * (t + T / 2));
                slot1[0] = make_uint4(bG1, bS1, bEU1, bEUL1);
                slot1[1] = make_uint4(bEUR1, bEL1, 0u, 0u);
            }
            hmax_p = hmax_c;
            hmin_p = hmin_c;
            hmax_c = hmax_n;
            hmin_c = hmin_n;
            Lp = Lc;
            vp = vc;
            Rp = Rc;
            vc = vn;
            Lc = Ln;
            Rc = Rn;
        }
        if (g.th == T) {
            // The window's high halves now hold rows T - 1 (p) and T (c).
            uint32_t lo;
            ballot_pair_eq(vp, Lc, lo, bEq[0]);
            ballot_pair_eq(vp, vc, lo, bEq[1]);
            ballot_pair_eq(vp, Rc, lo, bEq[2]);
        }
    }

    __syncwarp();
    {
        // Lane y takes row y's masks (rows beyond the tile stay 0) and clears
        // the words for the union-find.
        uint4* slot = reinterpret_cast<uint4*>(W + 8 * lane);
        if (lane < g.th) {
            const uint4 m0 = slot[0];
            const uint4 m1 = slot[1];
            const uint32_t cols = g.tw == T ? ~0u : (1u << g.tw) - 1u;
            rL = ~(m0.x & m0.y) & cols;   // not decided, inside the image
            rGT = rL & m0.x;
            rLT = rL & m0.y;
            rEU = m0.z;
            rEUL = m0.w;
            rEUR = m1.x;
            rEL = m1.y;
        }
        slot[0] = make_uint4(0u, 0u, 0u, 0u);
        slot[1] = make_uint4(0u, 0u, 0u, 0u);
    }

    // Staged pixel (x, y) of the tile, x and y in -1 .. T.
    auto px = [&](int x, int y) -> int {
        const int r = y + 1;
        return r < kSlotRows ? shalf[2 * (r * kHaloW + x + 1)]
                             : shalf[2 * ((r - T / 2) * kHaloW + x + 1) + 1];
    };

    // -- seam masks: border pixels with an equal neighbour outside the tile --
    // Per side and offset d = -1, 0, 1 along the side, the border pixels
    // equal to their neighbour across the side at offset d.  Top: row 0's
    // masks against the halo row (up-left, up, up-right); bottom: the
    // scan's last step; left: bits 0 of the rows' up-left / left masks and
    // one comparison with the halo pixel below-left; right: bits 31 of the
    // up-right masks and two comparisons with the halo column.  An equality
    // that involves a pixel outside the image means nothing (false in the
    // scan's masks, staged bits compared here), so every use is restricted
    // to listed pixels.
    uint32_t sT, sB, sLc, sRc;
    {
    uint32_t tEq[3], lEq[3], rEq[3];
    {
        const int y = lane;
        tEq[0] = __shfl_sync(~0u, rEUL, 0);
        tEq[1] = __shfl_sync(~0u, rEU, 0);
        tEq[2] = __shfl_sync(~0u, rEUR, 0);
        const int vl = px(0, y);
        const int vr = px(T - 1, y);
        lEq[0] = __ballot_sync(~0u, (rEUL & 1u) != 0u);
        lEq[1] = __ballot_sync(~0u, (rEL & 1u) != 0u);
        lEq[2] = __ballot_sync(~0u, px(-1, y + 1) == vl);
        rEq[0] = __ballot_sync(~0u, (rEUR >> 31) != 0u);
        rEq[1] = __ballot_sync(~0u, px(T, y) == vr);
        rEq[2] = __ballot_sync(~0u, px(T, y + 1) == vr);
    }
    if (lane == 0) {
        // Kept for the seam items at the end, out of the registers.
        uint4* e4 = reinterpret_cast<uint4*>(ax.eq);
        e4[0] = make_uint4(tEq[0], tEq[1], tEq[2], bEq[0]);
        e4[1] = make_uint4(bEq[1], bEq[2], lEq[0], lEq[1]);
        e4[2] = make_uint4(lEq[2], rEq[0], rEq[1], rEq[2]);
    }
    {
        // Adjacent pixels along each side that are equal (so in one zone
        // when both are listed): rows 0 and th - 1 (left neighbours),
        // columns 0 and 31 (upper neighbours).
        const uint32_t el_t = __shfl_sync(~0u, rEL, 0);
        const uint32_t el_b = __shfl_sync(~0u, rEL, g.th - 1);
        const uint32_t eu_l = __ballot_sync(~0u, (rEU & 1u) != 0u);
        const uint32_t eu_r = __ballot_sync(~0u, (rEU >> 31) != 0u);
        if (lane == 0) {
            reinterpret_cast<uint4*>(ax.eq)[3] =
                make_uint4(el_t, el_b, eu_l, eu_r);
        }
    }
    const uint32_t rows_in = g.th == T ? ~0u : (1u << g.th) - 1u;
    // Only the tile's own sides are seams.
    sT = ext_t ? (tEq[0] | tEq[1] | tEq[2]) : 0u;
    sB = ext_b ? (bEq[0] | bEq[1] | bEq[2]) : 0u;
    sLc = ext_l ? (lEq[0] | lEq[1] | lEq[2]) & rows_in : 0u;
    sRc = (ext_r && g.tw == T) ? (rEq[0] | rEq[1] | rEq[2]) & rows_in : 0u;
    }

    // -- per row (lane y): runs, seam and dead pixels --------------------------
    const int y = lane;
    // Shuffles run on every lane; lane 0 then drops the value it read back.
    uint32_t Lm1 = __shfl_up_sync(~0u, rL, 1);
    if (y == 0) {
        Lm1 = 0u;
    }
    uint32_t Lp1 = __shfl_down_sync(~0u, rL, 1);
    uint32_t EUp1 = __shfl_down_sync(~0u, rEU, 1);
    uint32_t EULp1 = __shfl_down_sync(~0u, rEUL, 1);
    uint32_t EURp1 = __shfl_down_sync(~0u, rEUR, 1);
    if (y + 1 >= g.th) {
        Lp1 = EUp1 = EULp1 = EURp1 = 0u;
    }
    const uint32_t cont = rEL & rL & (rL << 1);
    const uint32_t heads = rL & ~cont;
    const uint32_t ends = rL & ~(cont >> 1);
    const uint32_t seam =
        rL & ((y == 0 ? sT : 0u) | (y == T - 1 ? sB : 0u) |
              ((sLc >> y) & 1u) | (((sRc >> y) & 1u) << 31));
    uint32_t dead = (rEL & ~(rL << 1) & ~1u) | ((rEL >> 1) & ~(rL >> 1)) |
                    (EUp1 & ~Lp1) | ((EURp1 << 1) & ~(Lp1 << 1)) |
                    ((EULp1 >> 1) & ~(Lp1 >> 1));
    if (y > 0) {
        dead |= (rEU & ~Lm1) | (rEUL & ~(Lm1 << 1) & ~1u) |
                (rEUR & ~(Lm1 >> 1) & 0x7FFFFFFFu);
    }
    dead &= rL;

    // -- links: one union per contact of equal runs in rows y - 1 and y -------
    volatile uint32_t* vw = words;
    uint32_t linked = 0u;   // pixels of this row where a union touches a run
    {
        uint32_t headsm1 = __shfl_up_sync(~0u, heads, 1);
        if (y == 0) {
            headsm1 = 0u;
        }
        const uint32_t eqlU = rEU & rL & Lm1;
        const uint32_t eqlUL = rEUL & rL & (Lm1 << 1);
        const uint32_t eqlUR = rEUR & rL & (Lm1 >> 1);
        const uint32_t A = eqlU & ~eqlUL;            // partner (x, y - 1)
        const uint32_t B = heads & eqlUL;            // partner (x - 1, y - 1)
        const uint32_t C = ends & eqlUR & ~eqlU;     // partner (x + 1, y - 1)
        uint32_t m = A | B | C;
        // The partners in row y - 1 of row y's contacts, handed up a lane.
        uint32_t partners = __shfl_down_sync(~0u, A | (B >> 1) | (C << 1), 1);
        if (y == T - 1) {
            partners = 0u;
        }
        linked = m | partners;
        // A run's first contact (lowest column; a carry from the run's head
        // stops at it) makes the partner above its parent with a plain
        // store: the lane writes only its own row's still-zero words, and
        // the parent lies in the row above, so the forest keeps every root
        // the smallest word of its tree.
        const uint32_t first = ((((cont >> 1) & ~m) + heads) & m);
        {
            uint32_t f = first;
#pragma unroll 1
            while (f) {
                const int x = __ffs(f) - 1;
                f &= f - 1u;
                const int xp = ((A >> x) & 1u) ? x
                             : ((B >> x) & 1u) ? x - 1 : x + 1;
                const int p = wb + run_word(y, head_of(heads, x));
                vw[p] = with_parent(0u, p,
                                    wb + run_word(y - 1, head_of(headsm1, xp)));
            }
        }
        __syncwarp();
        // Every other contact: a union (a first contact that was A or B and
        // also C still owes its C union).
        uint32_t rest_ab = (A | B) & ~first;
        uint32_t rest_c = C & ~(first & ~(A | B));
        while (__any_sync(~0u, (rest_ab | rest_c) != 0u)) {
            const uint32_t rest = rest_ab | rest_c;
            if (rest) {
                const int x = __ffs(rest) - 1;
                const uint32_t bit = 1u << x;
                const int p = wb + run_word(y, head_of(heads, x));
                if (rest_ab & bit) {
                    const int xp = ((A >> x) & 1u) ? x : x - 1;
                    runion(words, p,
                           wb + run_word(y - 1, head_of(headsm1, xp)), err);
                }
                if (rest_c & bit) {
                    runion(words, p,
                           wb + run_word(y - 1, head_of(headsm1, x + 1)), err);
                }
                rest_ab &= ~bit;
                rest_c &= ~bit;
            }
        }
    }
    __syncwarp();

    if constexpr (Q == 4) {
        // -- the quadrants' inner sides ------------------------------------------
        // Every pair of equal 8-adjacent pixels of two quadrants: a decided
        // pixel makes the listed one's zone decided ("dead"); two listed
        // pixels have their runs united in the shared union-find (one union
        // per streak of such pairs along a side).  Each quadrant handles its
        // own pixels; pairs whose other pixel lies outside the tile belong
        // to the tile's sides.
        cta->lmask[q][y] = rL;
        cta->hmask[q][y] = heads;
        __syncthreads();
        // Quadrant pq's word of the run holding (pc, pr), and whether that
        // pixel is listed.
        auto partner = [&](int pq, int pr, int pc, bool& plisted) -> int {
            plisted = (cta->lmask[pq][pr] >> pc) & 1u;
            return plisted ? pq * T * T +
                                 run_word(pr, head_of(cta->hmask[pq][pr], pc))
                           : 0;
        };
        const uint4* e4 = reinterpret_cast<const uint4*>(ax.eq);
        const uint4 e0 = e4[0], e1 = e4[1], e2 = e4[2], e3 = e4[3];
        const uint32_t eqT[3] = {e0.x, e0.y, e0.z};
        const uint32_t eqB[3] = {e0.w, e1.x, e1.y};
        const uint32_t eqL[3] = {e1.z, e1.w, e2.x};
        const uint32_t eqR[3] = {e2.y, e2.z, e2.w};
        auto firsts_ = [](uint32_t c, uint32_t same) {
            return c & ~((c << 1) & same);
        };
        if (!ext_t || !ext_b) {
            // Top (row 0 against quadrant row 0's bottom rows) or bottom
            // (row 31 against quadrant row 1's top rows); lanes = columns.
            const bool top = !ext_t;
            const int row = top ? 0 : T - 1;
            const int prow = top ? T - 1 : 0;
            const int pbase = top ? 0 : 2;   // the partner quadrant row
            const uint32_t lrow = __shfl_sync(~0u, rL, row);
            const uint32_t hrow = __shfl_sync(~0u, heads, row);
            const uint32_t same = top ? e3.x : e3.y;   // row's left equality
            const uint32_t* eq = top ? eqT : eqB;
            uint32_t dd = 0u, ll = 0u;
#pragma unroll
            for (int d = -1; d <= 1; ++d) {
                const int xp = lane + d;
                int pq = -1, pc = xp;
                if (xp >= 0 && xp < T) {
                    pq = pbase + qx;
                } else if (xp < 0 && qx == 1) {
                    pq = pbase;
                    pc = T - 1;
                } else if (xp >= T && qx == 0 && two_cols) {
                    pq = pbase + 1;
                    pc = 0;
                }
                const bool cand = pq >= 0 && ((lrow >> lane) & 1u) &&
                                  ((eq[d + 1] >> lane) & 1u);
                bool pl = false;
                const int pw = cand ? partner(pq, prow, pc, pl) : 0;
                const uint32_t un = __ballot_sync(~0u, cand && pl);
                dd |= __ballot_sync(~0u, cand && !pl);
                ll |= un;
                if ((firsts_(un, same) >> lane) & 1u) {
                    runion(words, wb + run_word(row, head_of(hrow, lane)), pw,
                           err);
                }
            }
            if (y == row) {
                dead |= dd;
                linked |= ll;
            }
        }
        if (!ext_l || !ext_r) {
            // Left (column 0 against quadrant column 0's right column) or
            // right (column 31 against column 1's left column); lanes = rows.
            const bool left = !ext_l;
            const int col = left ? 0 : T - 1;
            const int pcol = left ? T - 1 : 0;
            const int pside = left ? 0 : 1;   // the partner quadrant column
            const uint32_t same = left ? e3.z : e3.w;  // column's up equality
            const uint32_t* eq = left ? eqL : eqR;
            const bool mine = (rL >> col) & 1u;
            uint32_t dd = 0u, ll = 0u;
#pragma unroll
            for (int d = -1; d <= 1; ++d) {
                const int yp = y + d;
                int pq = -1, pr = yp;
                if (yp >= 0 && yp < T) {
                    pq = 2 * qy + pside;
                } else if (yp < 0 && qy == 1) {
                    pq = pside;
                    pr = T - 1;
                } else if (yp >= T && qy == 0 && two_rows) {
                    pq = 2 + pside;
                    pr = 0;
                }
                const bool cand = pq >= 0 && mine && ((eq[d + 1] >> y) & 1u);
                bool pl = false;
                const int pw = cand ? partner(pq, pr, pcol, pl) : 0;
                const uint32_t un = __ballot_sync(~0u, cand && pl);
                dd |= __ballot_sync(~0u, cand && !pl);
                ll |= un;
                if ((firsts_(un, same) >> y) & 1u) {
                    runion(words, wb + run_word(y, head_of(heads, col)), pw,
                           err);
                }
            }
            const uint32_t bit_c = 1u << col;
            if ((dd >> y) & 1u) {
                dead |= bit_c;
            }
            if ((ll >> y) & 1u) {
                linked |= bit_c;
            }
        }
        dead &= rL;
        // Every union of the tile is in place before any flatten.
        __syncthreads();
    }

    // -- runs that are zones of their own ---------------------------------------
    // A run that no union touches is a whole zone; unless it touches a seam,
    // its verdict follows from its own pixels and the flatten, record and
    // verdict loops below leave it out (its word stays untouched; the border
    // record of such a pixel is never asked for, since no pixel outside the
    // tile is equal to it).
    const RunShape shape = run_shape(cont, heads, ends);
    const uint32_t c_open = clean_heads(shape, linked | seam);
    const uint32_t c_dead = clean_heads(shape, dead);
    const uint32_t c_gt = clean_heads(shape, rGT);
    const uint32_t c_lt = clean_heads(shape, rLT);
    const uint32_t loop_heads = heads & ~c_open;
    // Heads of runs that hold no dead pixel and not both a pixel with a
    // greater and one with a smaller neighbour.
    const uint32_t undecided = c_dead & (c_gt | c_lt);
    // Each run's own zone flags at its head (a dead pixel sets both flags).
    const uint32_t own_gt = heads & ~(c_gt & c_dead);
    const uint32_t own_lt = heads & ~(c_lt & c_dead);
    const uint32_t own_seam = heads & ~clean_heads(shape, seam);
    // Heads of the runs whose maxima / minima bytes are 255; spread over the
    // runs after the verdict loop.
    uint32_t hmax = c_open & c_dead & c_gt;
    uint32_t hmin = c_open & c_dead & c_lt;

    // -- the loop runs, dealt out evenly -----------------------------------------
    // The flatten and verdict loops below visit the runs of `loop_heads`.
    // Row by row (lane = row) they would take as many steps as the busiest
    // row has runs; instead the runs are listed once in the shared memory of
    // the staged tile (no longer read) and each step takes the next 32 of
    // them, whatever their rows.  Entry: row (bits 0-4), head (5-9), own
    // zone flags (10-12), "undecided" (13).  A tile with more runs than the
    // list holds (far beyond natural images) keeps the row-by-row order.
    // The verdicts of the settled runs and the pixels of the logged runs are
    // collected per row in shared memory (hm_rows, hn_rows, lv_rows).
    uint16_t* const list = reinterpret_cast<uint16_t*>(ax.img);
    uint32_t* const hm_rows = reinterpret_cast<uint32_t*>(ax.img) + kListCap / 2;
    uint32_t* const hn_rows = hm_rows + T;
    uint32_t* const lv_rows = hn_rows + T;
    hm_rows[y] = 0u;
    hn_rows[y] = 0u;
    lv_rows[y] = 0u;
    // The undecided runs come first in the list (the verdict loop visits
    // only them), the others after: one prefix over both counts (16 bits
    // each; a tile has at most 1,024 runs).
    uint32_t both = 0;
    const uint32_t at = warp_prefix(
        __popc(loop_heads & undecided) | (__popc(loop_heads & ~undecided) << 16),
        both);
    const uint32_t n_und = both & 0xFFFFu;
    const uint32_t n_list = n_und + (both >> 16);
    const bool listed = n_list <= static_cast<uint32_t>(kListCap);
    if (listed) {
        uint32_t r = loop_heads;
        uint32_t ku = at & 0xFFFFu;
        uint32_t ko = n_und + (at >> 16);
        while (r) {
            const int h = __ffs(r) - 1;
            r &= r - 1u;
            const uint32_t und = (undecided >> h) & 1u;
            list[und ? ku++ : ko++] = static_cast<uint16_t>(
                y | (h << 5) | (((own_gt >> h) & 1u) << 10) |
                (((own_lt >> h) & 1u) << 11) | (((own_seam >> h) & 1u) << 12) |
                (und << 13));
        }
    }
    // Steps of the two loops: 32 runs each, or the busiest row's runs.
    const int steps_all =
        listed ? static_cast<int>((n_list + 31u) >> 5)
               : static_cast<int>(__reduce_max_sync(~0u, __popc(loop_heads)));
    const int steps_und =
        listed ? static_cast<int>((n_und + 31u) >> 5)
               : static_cast<int>(
                     __reduce_max_sync(~0u, __popc(loop_heads & undecided)));
    __syncwarp();
    // The run a lane takes at step `it`: from the list, or the next of its
    // row's runs in `r` (row order).  Returns false when it has none.
    auto take = [&](int it, uint32_t lim, uint32_t& r, int& yy, int& h,
                    uint32_t& own, bool& und) -> bool {
        if (listed) {
            const uint32_t idx = static_cast<uint32_t>(it * 32 + lane);
            if (idx >= lim) {
                return false;
            }
            const uint32_t e = list[idx];
            yy = static_cast<int>(e & 31u);
            h = static_cast<int>((e >> 5) & 31u);
            own = (e >> 10) & 7u;
            und = (e >> 13) & 1u;
            return true;
        }
        if (!r) {
            return false;
        }
        h = __ffs(r) - 1;
        r &= r - 1u;
        yy = y;
        own = ((own_gt >> h) & 1u) * kHasGreater |
              ((own_lt >> h) & 1u) * kHasSmaller |
              ((own_seam >> h) & 1u) * kTouchesSeam;
        und = (undecided >> h) & 1u;
        return true;
    };

    // -- flatten; zone flags ORed into the roots --------------------------------
    {
        uint32_t r = loop_heads;
#pragma unroll 1
        for (int it = 0; it < steps_all; ++it) {
            int yy = 0, h = 0;
            uint32_t own = 0u;
            bool und = false;
            if (take(it, n_list, r, yy, h, own, und)) {
                const int p = wb + run_word(yy, h);
                // The walk keeps the root's word: the flags read from it may
                // lag other lanes' ORs, which only costs a redundant OR.
                const uint32_t wp = vw[p];
                uint32_t wr = wp;
                int root = p;
#pragma unroll 1
                for (int k = 0; k < kWalkBound; ++k) {
                    const int up = rparent(wr, root);
                    if (up == root) break;
                    root = up;
                    wr = vw[root];
                }
                if (root != p) {
                    // p is not a root: no other lane writes its word now.
                    vw[p] = with_parent(wp, p, root);
                }
                const uint32_t zf = (wr >> kZoneShift) & 7u;
                if ((zf & own) != own) {
                    atomicOr(words + root, own << kZoneShift);
                }
            }
        }
    }
    // Zone flags are complete at every root (of any quadrant) from here on.
    if constexpr (Q == 4) {
        __syncthreads();
    } else {
        __syncwarp();
    }

    // -- listed pixels: verdicts of settled zones, run log of live zones ------
    // `hm_rows` / `hn_rows` collect the heads of the runs of settled zones
    // whose maxima / minima byte is 255.  A live seam zone gets its record
    // (fragment) when the loop first meets one of its runs: one lane per
    // root takes the next number, in the order of the loop's steps and
    // lanes.
    uint32_t* plog = a.pending + item * kPendingT;
    int nlog = 0;
    uint32_t live_px = 0u;   // pixels of this lane's logged runs
    uint32_t nrec = 0;
    const int64_t frag_base = item * kSlotsT;
    if constexpr (Q == 1) {
        // Runs that hold a dead pixel, or both a pixel with a greater and
        // one with a smaller neighbour, are in a decided zone: 0 in both
        // masks, nothing to log; only the other runs are visited.
        uint32_t r = loop_heads & undecided;
#pragma unroll 1
        for (int it = 0; it < steps_und; ++it) {
            bool live = false;
            int h = 0, yy = 0, root = 0;
            uint32_t rec1 = 0u;
            uint32_t own = 0u;
            bool und = false;
            if (take(it, n_und, r, yy, h, own, und) && und) {
                const int p = wb + run_word(yy, h);
                root = rparent(vw[p], p);
                const uint32_t w = vw[root];
                const uint32_t z = (w >> kZoneShift) & 7u;
                live = (z & kTouchesSeam) && (z & kDead) != kDead;
                if (live) {
                    rec1 = (w >> kRecShift) & 0xFFu;
                } else {
                    if (!(z & kHasGreater)) {
                        atomicOr(hm_rows + yy, 1u << h);
                    }
                    if (!(z & kHasSmaller)) {
                        atomicOr(hn_rows + yy, 1u << h);
                    }
                }
            }
            const bool need = live && rec1 == 0u;
            if (__any_sync(~0u, need)) {
                // Lanes on the same new root: the lowest one numbers it.
                const uint32_t same =
                    __match_any_sync(~0u, need ? root : -1 - lane);
                const int leader = __ffs(same) - 1;
                const bool lead = need && leader == lane;
                const uint32_t leads = __ballot_sync(~0u, lead);
                uint32_t mine = 0u;
                if (lead) {
                    const uint32_t rec = nrec + __popc(leads & lt_mask);
                    if (rec < static_cast<uint32_t>(kSlotsT)) {
                        const uint32_t w = vw[root];
                        vw[root] = w | ((rec + 1u) << kRecShift);
                        const uint32_t z = (w >> kZoneShift) & 3u;
                        const int64_t gi = frag_base + rec;
                        a.parent[gi] = static_cast<int32_t>(gi);
                        a.bits[gi] = z | (z << kLocalShift);
                        mine = rec + 1u;
                    } else {
                        err = kErrFragmentOverflow;
                    }
                }
                const uint32_t got = __shfl_sync(~0u, mine, leader);
                if (need) {
                    rec1 = got;
                }
                nrec += __popc(leads);
                __syncwarp();
            }
            // The run's end, from its row's run ends.
            const uint32_t ends_yy = __shfl_sync(~0u, ends, yy);
            bool logged = false;
            uint32_t entry = 0u;
            if (live && rec1) {
                const int e = __ffs(ends_yy & ~((1u << h) - 1u)) - 1;
                logged = true;
                entry = pending_entry(static_cast<int>(rec1 - 1u), h, yy,
                                      e - h + 1);
                live_px += static_cast<uint32_t>(e - h + 1);
                atomicOr(lv_rows + yy, ((2u << e) - 1u) & ~((1u << h) - 1u));
                // The run's own head word also carries the record (a root's
                // already does; other head words have these bits free, and
                // only this lane touches this run's word).
                const int p = wb + run_word(yy, h);
                if (p != root) {
                    vw[p] |= rec1 << kRecShift;
                }
            }
            const uint32_t bal = __ballot_sync(~0u, logged);
            if (logged) {
                plog[nlog + __popc(bal & lt_mask)] = entry;
            }
            nlog += __popc(bal);
        }
    } else {
        // Tile edge 64: a zone's root may lie in another quadrant, met by
        // another warp, so records go to the roots first (each root is met
        // once, at its own run; the tile's counter numbers them), then every
        // run reads its root.
        {
            uint32_t r = loop_heads;
#pragma unroll 1
            for (int it = 0; it < steps_all; ++it) {
                int yy = 0, h = 0, p = 0;
                uint32_t own = 0u, w = 0u;
                bool und = false;
                bool live_root = false;
                if (take(it, n_list, r, yy, h, own, und)) {
                    p = wb + run_word(yy, h);
                    w = vw[p];
                    const uint32_t z = (w >> kZoneShift) & 7u;
                    live_root = rparent(w, p) == p && (z & kTouchesSeam) &&
                                (z & kDead) != kDead;
                }
                const uint32_t roots = __ballot_sync(~0u, live_root);
                if (roots) {
                    uint32_t base = 0u;
                    if (lane == 0) {
                        base = atomicAdd(&cta->nrec, __popc(roots));
                    }
                    base = __shfl_sync(~0u, base, 0);
                    if (live_root) {
                        const uint32_t rec = base + __popc(roots & lt_mask);
                        if (rec < static_cast<uint32_t>(kSlotsT)) {
                            vw[p] = w | ((rec + 1u) << kRecShift);
                            const uint32_t z = (w >> kZoneShift) & 3u;
                            const int64_t gi = frag_base + rec;
                            a.parent[gi] = static_cast<int32_t>(gi);
                            a.bits[gi] = z | (z << kLocalShift);
                        } else {
                            err = kErrFragmentOverflow;
                        }
                    }
                }
            }
        }
        __syncthreads();
        uint32_t r = loop_heads & undecided;
#pragma unroll 1
        for (int it = 0; it < steps_und; ++it) {
            bool logged = false;
            int h = 0, yy = 0, p = 0, root = 0;
            uint32_t rec1 = 0u;
            uint32_t own = 0u;
            bool und = false;
            if (take(it, n_und, r, yy, h, own, und) && und) {
                p = wb + run_word(yy, h);
                root = rparent(vw[p], p);
                const uint32_t w = vw[root];
                const uint32_t z = (w >> kZoneShift) & 7u;
                if ((z & kTouchesSeam) && (z & kDead) != kDead) {
                    rec1 = (w >> kRecShift) & 0xFFu;
                    logged = rec1 != 0u;   // 0: the tile ran out of records
                } else {
                    if (!(z & kHasGreater)) {
                        atomicOr(hm_rows + yy, 1u << h);
                    }
                    if (!(z & kHasSmaller)) {
                        atomicOr(hn_rows + yy, 1u << h);
                    }
                }
            }
            const uint32_t ends_yy = __shfl_sync(~0u, ends, yy);
            uint32_t entry = 0u;
            if (logged) {
                const int e = __ffs(ends_yy & ~((1u << h) - 1u)) - 1;
                entry = pending_entry(static_cast<int>(rec1 - 1u), T * qx + h,
                                      T * qy + yy, e - h + 1);
                live_px += static_cast<uint32_t>(e - h + 1);
                atomicOr(lv_rows + yy, ((2u << e) - 1u) & ~((1u << h) - 1u));
                if (p != root) {
                    vw[p] |= rec1 << kRecShift;
                }
            }
            const uint32_t bal = __ballot_sync(~0u, logged);
            if (bal) {
                uint32_t base = 0u;
                if (lane == 0) {
                    base = atomicAdd(&cta->nlog, __popc(bal));
                }
                base = __shfl_sync(~0u, base, 0);
                if (logged) {
                    plog[base + __popc(bal & lt_mask)] = entry;
                }
            }
        }
    }
    __syncwarp();
    hmax |= hm_rows[y];
    hmin |= hn_rows[y];
    const uint32_t live_row = lv_rows[y];   // pixels of this row's logged runs
    const uint32_t vmax = run_span(shape, hmax);
    const uint32_t vmin = run_span(shape, hmin);
    // The tile's logged pixels (a statistic: bits 16-31 of its log count).
    const uint32_t logged_px = __reduce_add_sync(~0u, live_px);
    // The mask bytes of every pixel of the tile.  Pixels of live zones get a
    // placeholder 0 in both masks here; the resolve pass, which runs after
    // this pass, rewrites those of zones that end up in a mask (most end up
    // in neither, and their placeholders are final).  So whole rows are
    // written, with 16-, 8- or 4-byte stores where the output rows allow it.
    {
        const uint64_t bmx = reinterpret_cast<uint64_t>(
            omax + static_cast<int64_t>(g.y0) * out_pitch + g.x0);
        const uint64_t bmn = reinterpret_cast<uint64_t>(
            omin + static_cast<int64_t>(g.y0) * out_pitch + g.x0);
        const uint64_t align = bmx | bmn | static_cast<uint64_t>(out_pitch);
        int vec = (align & 15u) == 0 ? 16 : (align & 7u) == 0 ? 8
                : (align & 3u) == 0 ? 4 : 1;
        if (g.tw < T || g.th < T) {
            vec = 1;
        }
        if (vec == 16) {
            store_rows<16>(omax, omin, g, out_pitch, vmax, vmin);
        } else if (vec == 8) {
            store_rows<8>(omax, omin, g, out_pitch, vmax, vmin);
        } else if (vec == 4) {
            store_rows<4>(omax, omin, g, out_pitch, vmax, vmin);
        } else {
            uint8_t* pmx = omax + static_cast<int64_t>(g.y0) * out_pitch +
                           g.x0 + lane;
            uint8_t* pmn = omin + static_cast<int64_t>(g.y0) * out_pitch +
                           g.x0 + lane;
#pragma unroll 2
            for (int yy = 0; yy < g.th; ++yy) {
                const uint32_t mxr = __shfl_sync(~0u, vmax, yy);
                const uint32_t mnr = __shfl_sync(~0u, vmin, yy);
                if (col_ok) {
                    *pmx = ((mxr >> lane) & 1u) ? 255 : 0;
                    *pmn = ((mnr >> lane) & 1u) ? 255 : 0;
                }
                pmx += out_pitch;
                pmn += out_pitch;
            }
        }
    }

    // -- border records, seam items ---------------------------------------------
    // Border record of every side pixel: its zone's record if the zone is
    // live (then one of its runs was logged, and the run's head word holds
    // the record), else "dead": a pixel equal to a pixel across the seam is
    // in a zone touching the seam, so it is live or decided.
    uint8_t* border = a.border + item * kSlotsT;
    auto rec_at = [&](int x, int yy, uint32_t hrow) -> uint32_t {
        const uint32_t w = vw[wb + run_word(yy, head_of(hrow, x))];
        return ((w >> kRecShift) & 0xFFu) - 1u;
    };
    const uint32_t live_t = __shfl_sync(~0u, live_row, 0);
    const uint32_t heads_t = __shfl_sync(~0u, heads, 0);
    const uint32_t live_b0 = __shfl_sync(~0u, live_row, g.th - 1);
    const uint32_t heads_b = __shfl_sync(~0u, heads, g.th - 1);
    const uint32_t live_l = __ballot_sync(~0u, (live_row & 1u) != 0u);
    const int last_col = max(g.tw - 1, 0);
    const uint32_t live_r0 =
        __ballot_sync(~0u, ((live_row >> last_col) & 1u) != 0u);
    const uint32_t bit = 1u << lane;
    const uint32_t rt = (live_t & bit) ? rec_at(lane, 0, heads_t) : kDeadRecord;
    const uint32_t rb =
        (live_b0 & bit) ? rec_at(lane, g.th - 1, heads_b) : kDeadRecord;
    const uint32_t rl = (live_row & 1u) ? rec_at(0, y, heads) : kDeadRecord;
    const uint32_t rr = ((live_row >> last_col) & 1u)
                            ? rec_at(last_col, y, heads) : kDeadRecord;
    // Border record arrays: top, bottom, left, right, TT each (positions
    // along the tile's side).
    if (lane < g.tw) {
        if (ext_t) {
            border[T * qx + lane] = static_cast<uint8_t>(rt);
        }
        if (ext_b) {
            border[TT + T * qx + lane] = static_cast<uint8_t>(rb);
        }
    }
    if (lane < g.th) {
        if (ext_l) {
            border[2 * TT + T * qy + lane] = static_cast<uint8_t>(rl);
        }
        if (ext_r) {
            border[3 * TT + T * qy + lane] = static_cast<uint8_t>(rr);
        }
    }
    // Seam items: one per equal pair (live pixel here, pixel across the
    // seam at offset d), except that of a streak of such pairs in one
    // direction whose pixels here are adjacent and in one zone (so are
    // their partners, adjacent and equal: one zone in one neighbour tile)
    // only the first is kept.  Lanes are the positions along the side.
    uint32_t* items = a.seam_items + item * kSeamT;
    int nitems = 0;
    auto emit = [&](uint32_t m, uint32_t rec, int dir, int off) {
        if (!m) {
            return;
        }
        uint32_t base = static_cast<uint32_t>(nitems);
        if constexpr (Q == 4) {
            if (lane == 0) {
                base = atomicAdd(&cta->nitems, __popc(m));
            }
            base = __shfl_sync(~0u, base, 0);
        }
        if (m & bit) {
            items[base + __popc(m & lt_mask)] =
                rec | (static_cast<uint32_t>(off) << 8) |
                (static_cast<uint32_t>(dir) << 16);
        }
        nitems += __popc(m);
    };
    // Keeps the first pair of every streak: c are the candidate positions,
    // same the positions whose pixel is in the zone of the previous one.
    auto firsts = [](uint32_t c, uint32_t same) {
        return c & ~((c << 1) & same);
    };
    uint32_t qT[3], qB[3], qL[3], qR[3], el_t, el_b, eu_l, eu_r;
    {
        const uint4* e4 = reinterpret_cast<const uint4*>(ax.eq);
        const uint4 e0 = e4[0], e1 = e4[1], e2 = e4[2], e3 = e4[3];
        el_t = e3.x;
        el_b = e3.y;
        eu_l = e3.z;
        eu_r = e3.w;
        qT[0] = e0.x; qT[1] = e0.y; qT[2] = e0.z;
        qB[0] = e0.w; qB[1] = e1.x; qB[2] = e1.y;
        qL[0] = e1.z; qL[1] = e1.w; qL[2] = e2.x;
        qR[0] = e2.y; qR[1] = e2.z; qR[2] = e2.w;
    }
    // Only the tile's own sides have seam items, and only where a
    // neighbour tile lies across them.
    const uint32_t live_tt = ext_t ? live_t : 0u;
    const uint32_t live_ll = ext_l ? live_l : 0u;
    const uint32_t live_b =
        (ext_b && tg.th == TT && tg.y0 + TT < height) ? live_b0 : 0u;
    const uint32_t live_r =
        (ext_r && tg.tw == TT && tg.x0 + TT < width) ? live_r0 : 0u;
    if (live_tt | live_b) {
#pragma unroll
        for (int d = -1; d <= 1; ++d) {
            // The direction changes between tile positions 0 and 1 (d = -1)
            // or TT - 2 and TT - 1 (d = 1): a streak does not continue
            // across it.
            const uint32_t cont =
                d < 0 ? (qx == 0 ? ~2u : ~0u)
                      : (d > 0 ? (T * qx + T == TT ? 0x7FFFFFFFu : ~0u)
                               : ~0u);
            const int x2 = T * qx + lane + d;
            const int side_off = x2 < 0 ? TT - 1 : (x2 >= TT ? 0 : x2);
            if (live_tt) {
                emit(firsts(live_tt & qT[d + 1], el_t & cont), rt,
                     x2 < 0 ? kRelTopLeft : (x2 >= TT ? kRelTopRight : kRelTop),
                     TT + side_off);
            }
            if (live_b) {
                emit(firsts(live_b & qB[d + 1], el_b & cont), rb,
                     x2 < 0 ? kRelBottomLeft
                            : (x2 >= TT ? kRelBottomRight : kRelBottom),
                     side_off);
            }
        }
    }
    if (live_ll | live_r) {
        // Partners inside the tile's row band only (the corners belong to
        // the top and bottom sides).
#pragma unroll
        for (int d = -1; d <= 1; ++d) {
            // Rows y of this square whose partner row T qy + y + d lies in
            // 0 .. tile height - 1.
            const int lo = max(0, -d - T * qy);
            const int hi = min(T, tg.th - d - T * qy);
            const uint32_t band =
                hi > lo ? ((hi >= 32 ? ~0u : (1u << hi) - 1u) & ~((1u << lo) - 1u))
                        : 0u;
            if (live_ll) {
                emit(firsts(live_ll & qL[d + 1] & band, eu_l), rl, kRelLeft,
                     3 * TT + T * qy + y + d);
            }
            if (live_r) {
                emit(firsts(live_r & qR[d + 1] & band, eu_r), rr, kRelRight,
                     2 * TT + T * qy + y + d);
            }
        }
    }
    if constexpr (Q == 1) {
        if (lane == 0) {
            a.fragment_count[item] = static_cast<uint16_t>(
                min(nrec, static_cast<uint32_t>(kSlotsT)));
            a.pending_count[item] =
                static_cast<uint32_t>(nlog) | (logged_px << 16);
            a.seam_count[item] = static_cast<uint32_t>(nitems);
        }
    } else {
        if (lane == 0 && logged_px) {
            atomicAdd(&cta->logged_px, logged_px);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            a.fragment_count[item] = static_cast<uint16_t>(
                min(cta->nrec, static_cast<uint32_t>(kSlotsT)));
            a.pending_count[item] = cta->nlog | (cta->logged_px << 16);
            a.seam_count[item] = cta->nitems;
        }
    }
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(item));
    }
}

}  // namespace rowscan

}  // namespace ss

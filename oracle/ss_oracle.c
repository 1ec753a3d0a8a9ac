/*
 * ss_oracle.c -- CPU oracle for the exact dual regional-extrema route.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file: it is the checker that the parity tests, the smoke check and
 * the CPU-baseline leg of the benchmark compare the CUDA path against.
 *
 * Semantic rule (the one the reference's golden masks were made with,
 * oracles/build_oracle_v0_1.m:109-110, MATLAB imregionalmax/imregionalmin with
 * 8-connectivity):
 *   - a "flat zone" is an 8-connected set of equal-valued pixels;
 *   - a pixel belongs to the regional-maximum mask iff no pixel of its flat
 *     zone has a strictly greater 8-neighbour; likewise for the minimum mask
 *     with "strictly smaller";
 *   - pixels outside the image are absent (not -inf / +inf), so a constant
 *     image is one maximum and one minimum at the same time;
 *   - masks are bytes, 255 inside the set and 0 outside.
 *
 * Three independent routes are provided:
 *   ss_oracle_floodfill  -- breadth-first flood fill per flat zone, following
 *                           datasets/bbbc038_distance/
 *                           derive_bbbc038_distance_markers_v0_2.py:61-105
 *                           (foreground = whole image, plus a has_smaller flag).
 *   ss_oracle_unionfind  -- dense per-pixel union-find over the four backward
 *                           equal edges with per-pixel greater/smaller flags
 *                           reduced at the root, following the Global-UF route
 *                           harness/primary/snapshot_gpu_benchmark_globaluf_
 *                           ole_v0_1.cu:105-179 (flags, reduce, materialize)
 *                           and :185-259 (init, union, compress).
 *   ss_oracle_bands      -- the same union-find split into row bands that
 *                           run on separate OpenMP threads and are merged at
 *                           band seams; the timed CPU baseline for one large
 *                           image.
 * plus
 *   ss_oracle_batch      -- one image per OpenMP thread (union-find route);
 *                           the timed CPU baseline for an image corpus.
 *   ss_oracle_tile_fragments -- per T x T tile, the number of tile-local flat
 *                           zones that have an equal 8-neighbour outside the
 *                           tile; the quantity the reference stores in
 *                           tile_fragment_counts (harness/primary/
 *                           snapshot_sparse_seam_cuda_v1_0.cu:395-410, 446-449,
 *                           summed into active_fragments at :852-863).
 *
 * All routes return 0 on success and a negative value on invalid arguments or
 * allocation failure.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SS_HAS_GREATER 1u
#define SS_HAS_SMALLER 2u

static int bad_geometry(int w, int h, long pitch, long out_pitch) {
    return w <= 0 || h <= 0 || pitch < w || out_pitch < w;
}

/* ------------------------------------------------------------------------ */
/* Flood fill                                                                */
/* ------------------------------------------------------------------------ */

int ss_oracle_floodfill(const uint8_t* img, int w, int h, long pitch,
                        uint8_t* maxima, uint8_t* minima, long out_pitch) {
    if (!img || !maxima || !minima || bad_geometry(w, h, pitch, out_pitch)) {
        return -1;
    }
    const long n = (long)w * (long)h;
    uint8_t* visited = (uint8_t*)calloc((size_t)n, 1);
    int32_t* queue = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    if (!visited || !queue) {
        free(visited);
        free(queue);
        return -2;
    }
    for (long start = 0; start < n; ++start) {
        if (visited[start]) {
            continue;
        }
        const int sx = (int)(start % w);
        const int sy = (int)(start / w);
        const uint8_t value = img[(long)sy * pitch + sx];
        /* The queue doubles as the zone's pixel list: everything pushed for
         * this zone sits in queue[0, tail). */
        long head = 0;
        long tail = 0;
        queue[tail++] = (int32_t)start;
        visited[start] = 1;
        int has_greater = 0;
        int has_smaller = 0;
        while (head < tail) {
            const int32_t p = queue[head++];
            const int x = p % w;
            const int y = p / w;
            for (int dy = -1; dy <= 1; ++dy) {
                const int ny = y + dy;
                if (ny < 0 || ny >= h) {
                    continue;
                }
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = x + dx;
                    if ((dx == 0 && dy == 0) || nx < 0 || nx >= w) {
                        continue;
                    }
                    const uint8_t nv = img[(long)ny * pitch + nx];
                    if (nv > value) {
                        has_greater = 1;
                    } else if (nv < value) {
                        has_smaller = 1;
                    } else {
                        const long q = (long)ny * w + nx;
                        if (!visited[q]) {
                            visited[q] = 1;
                            queue[tail++] = (int32_t)q;
                        }
                    }
                }
            }
        }
        const uint8_t mx = has_greater ? 0 : 255;
        const uint8_t mn = has_smaller ? 0 : 255;
        for (long i = 0; i < tail; ++i) {
            const int x = queue[i] % w;
            const int y = queue[i] / w;
            maxima[(long)y * out_pitch + x] = mx;
            minima[(long)y * out_pitch + x] = mn;
        }
    }
    free(visited);
    free(queue);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Dense union-find                                                          */
/* ------------------------------------------------------------------------ */

static int32_t uf_find(const int32_t* parent, int32_t node) {
    while (parent[node] != node) {
        node = parent[node];
    }
    return node;
}

/* Links the larger root below the smaller one, so every link points to a
 * smaller index and the final root of a set is its smallest member. */
static void uf_union(int32_t* parent, int32_t a, int32_t b) {
    int32_t ra = uf_find(parent, a);
    int32_t rb = uf_find(parent, b);
    if (ra == rb) {
        return;
    }
    if (ra < rb) {
        parent[rb] = ra;
    } else {
        parent[ra] = rb;
    }
}

/* Per-pixel greater/smaller flags over the valid 8-neighbourhood. */
static uint8_t pixel_flags(const uint8_t* img, int w, int h, long pitch,
                           int x, int y) {
    const uint8_t v = img[(long)y * pitch + x];
    uint8_t f = 0;
    for (int dy = -1; dy <= 1; ++dy) {
        const int ny = y + dy;
        if (ny < 0 || ny >= h) {
            continue;
        }
        for (int dx = -1; dx <= 1; ++dx) {
            const int nx = x + dx;
            if ((dx == 0 && dy == 0) || nx < 0 || nx >= w) {
                continue;
            }
            const uint8_t nv = img[(long)ny * pitch + nx];
            f |= nv > v ? SS_HAS_GREATER : 0u;
            f |= nv < v ? SS_HAS_SMALLER : 0u;
        }
    }
    return f;
}

/* Unions the backward equal edges (left, up, up-left, up-right) of rows
 * [y_begin, y_end); edges into row y_begin - 1 are included only when
 * include_top is set. */
static void union_rows(const uint8_t* img, int w, long pitch, int32_t* parent,
                       int y_begin, int y_end, int include_top) {
    for (int y = y_begin; y < y_end; ++y) {
        const uint8_t* row = img + (long)y * pitch;
        const uint8_t* up = row - pitch;
        const int up_ok = y > 0 && (y > y_begin || include_top);
        for (int x = 0; x < w; ++x) {
            const int32_t i = (int32_t)((long)y * w + x);
            const uint8_t v = row[x];
            if (x > 0 && row[x - 1] == v) {
                uf_union(parent, i, i - 1);
            }
            if (up_ok) {
                if (up[x] == v) {
                    uf_union(parent, i, i - w);
                }
                if (x > 0 && up[x - 1] == v) {
                    uf_union(parent, i, i - w - 1);
                }
                if (x + 1 < w && up[x + 1] == v) {
                    uf_union(parent, i, i - w + 1);
                }
            }
        }
    }
}

static void materialize_rows(const uint8_t* img, int w, int h, long pitch,
                             const int32_t* parent, const uint8_t* root_flags,
                             uint8_t* maxima, uint8_t* minima, long out_pitch,
                             int y_begin, int y_end) {
    (void)img;
    (void)h;
    (void)pitch;
    for (int y = y_begin; y < y_end; ++y) {
        for (int x = 0; x < w; ++x) {
            const int32_t i = (int32_t)((long)y * w + x);
            const uint8_t f = root_flags[parent[i]];
            maxima[(long)y * out_pitch + x] = (f & SS_HAS_GREATER) ? 0 : 255;
            minima[(long)y * out_pitch + x] = (f & SS_HAS_SMALLER) ? 0 : 255;
        }
    }
}

int ss_oracle_unionfind(const uint8_t* img, int w, int h, long pitch,
                        uint8_t* maxima, uint8_t* minima, long out_pitch) {
    if (!img || !maxima || !minima || bad_geometry(w, h, pitch, out_pitch)) {
        return -1;
    }
    const long n = (long)w * (long)h;
    if (n > 0x7fffffffL) {
        return -1;
    }
    int32_t* parent = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    uint8_t* root_flags = (uint8_t*)calloc((size_t)n, 1);
    if (!parent || !root_flags) {
        free(parent);
        free(root_flags);
        return -2;
    }
    for (long i = 0; i < n; ++i) {
        parent[i] = (int32_t)i;
    }
    union_rows(img, w, pitch, parent, 0, h, 1);
    for (long i = 0; i < n; ++i) {
        parent[i] = uf_find(parent, (int32_t)i);
    }
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const long i = (long)y * w + x;
            root_flags[parent[i]] |= pixel_flags(img, w, h, pitch, x, y);
        }
    }
    materialize_rows(img, w, h, pitch, parent, root_flags, maxima, minima,
                     out_pitch, 0, h);
    free(parent);
    free(root_flags);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Row-band parallel union-find (CPU baseline for one large image)           */
/* ------------------------------------------------------------------------ */

int ss_oracle_bands(const uint8_t* img, int w, int h, long pitch,
                    uint8_t* maxima, uint8_t* minima, long out_pitch,
                    int threads) {
    if (!img || !maxima || !minima || bad_geometry(w, h, pitch, out_pitch)) {
        return -1;
    }
    const long n = (long)w * (long)h;
    if (n > 0x7fffffffL) {
        return -1;
    }
    if (threads < 1) {
        threads = 1;
    }
    if (threads > h) {
        threads = h;
    }
    int32_t* parent = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    int32_t* label = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    uint8_t* root_flags = (uint8_t*)calloc((size_t)n, 1);
    if (!parent || !label || !root_flags) {
        free(parent);
        free(label);
        free(root_flags);
        return -2;
    }
    const int bands = threads;
    /* Phase 1: each band labels its own rows; links never leave the band. */
#pragma omp parallel for num_threads(threads) schedule(static, 1)
    for (int b = 0; b < bands; ++b) {
        const int y0 = (int)((long)h * b / bands);
        const int y1 = (int)((long)h * (b + 1) / bands);
        for (long i = (long)y0 * w; i < (long)y1 * w; ++i) {
            parent[i] = (int32_t)i;
        }
        union_rows(img, w, pitch, parent, y0, y1, 0);
    }
    /* Phase 2: serial merge across band seams (first row of each band with
     * the last row of the band above). */
    for (int b = 1; b < bands; ++b) {
        const int y = (int)((long)h * b / bands);
        const uint8_t* row = img + (long)y * pitch;
        const uint8_t* up = row - pitch;
        for (int x = 0; x < w; ++x) {
            const int32_t i = (int32_t)((long)y * w + x);
            const uint8_t v = row[x];
            if (up[x] == v) {
                uf_union(parent, i, i - w);
            }
            if (x > 0 && up[x - 1] == v) {
                uf_union(parent, i, i - w - 1);
            }
            if (x + 1 < w && up[x + 1] == v) {
                uf_union(parent, i, i - w + 1);
            }
        }
    }
    /* Phase 3: flatten into a separate label array (the forest is read-only
     * here, so the threads share it without synchronisation). */
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const long i = (long)y * w + x;
            label[i] = uf_find(parent, (int32_t)i);
        }
    }
    /* Phase 4: per-pixel flags OR-reduced into the root. */
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const long i = (long)y * w + x;
            const uint8_t f = pixel_flags(img, w, h, pitch, x, y);
            uint8_t* slot = &root_flags[label[i]];
            if (f && (__atomic_load_n(slot, __ATOMIC_RELAXED) & f) != f) {
                __atomic_fetch_or(slot, f, __ATOMIC_RELAXED);
            }
        }
    }
    /* Phase 5: materialize. */
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int y = 0; y < h; ++y) {
        materialize_rows(img, w, h, pitch, label, root_flags, maxima, minima,
                         out_pitch, y, y + 1);
    }
    free(parent);
    free(label);
    free(root_flags);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Corpus: one image per thread                                              */
/* ------------------------------------------------------------------------ */

int ss_oracle_batch(int count, const uint8_t* const* images, const int* widths,
                    const int* heights, const long* pitches,
                    uint8_t* const* maxima, uint8_t* const* minima,
                    const long* out_pitches, int threads) {
    if (count < 0 || (count > 0 && (!images || !widths || !heights ||
                                    !pitches || !maxima || !minima ||
                                    !out_pitches))) {
        return -1;
    }
    if (threads < 1) {
        threads = 1;
    }
    int failures = 0;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1) \
    reduction(+ : failures)
    for (int i = 0; i < count; ++i) {
        failures += ss_oracle_unionfind(images[i], widths[i], heights[i],
                                        pitches[i], maxima[i], minima[i],
                                        out_pitches[i]) != 0;
    }
    return failures ? -3 : 0;
}

/* ------------------------------------------------------------------------ */
/* Tile-local seam fragments (statistics pin)                                */
/* ------------------------------------------------------------------------ */

int ss_oracle_tile_fragments(const uint8_t* img, int w, int h, long pitch,
                             int tile, uint16_t* counts) {
    if (!img || !counts || tile < 1 || bad_geometry(w, h, pitch, w)) {
        return -1;
    }
    const int tiles_x = (w + tile - 1) / tile;
    const int tiles_y = (h + tile - 1) / tile;
    const int tp = tile * tile;
    uint8_t* visited = (uint8_t*)malloc((size_t)tp);
    int32_t* queue = (int32_t*)malloc((size_t)tp * sizeof(int32_t));
    if (!visited || !queue) {
        free(visited);
        free(queue);
        return -2;
    }
    for (int ty = 0; ty < tiles_y; ++ty) {
        for (int tx = 0; tx < tiles_x; ++tx) {
            const int x0 = tx * tile;
            const int y0 = ty * tile;
            const int tw = w - x0 < tile ? w - x0 : tile;
            const int th = h - y0 < tile ? h - y0 : tile;
            memset(visited, 0, (size_t)tp);
            int fragments = 0;
            for (int s = 0; s < tw * th; ++s) {
                if (visited[s]) {
                    continue;
                }
                const uint8_t v =
                    img[(long)(y0 + s / tw) * pitch + x0 + s % tw];
                long head = 0;
                long tail = 0;
                queue[tail++] = s;
                visited[s] = 1;
                int touches_seam = 0;
                while (head < tail) {
                    const int p = queue[head++];
                    const int lx = p % tw;
                    const int ly = p / tw;
                    for (int dy = -1; dy <= 1; ++dy) {
                        for (int dx = -1; dx <= 1; ++dx) {
                            if (dx == 0 && dy == 0) {
                                continue;
                            }
                            const int gx = x0 + lx + dx;
                            const int gy = y0 + ly + dy;
                            if (gx < 0 || gx >= w || gy < 0 || gy >= h) {
                                continue;
                            }
                            if (img[(long)gy * pitch + gx] != v) {
                                continue;
                            }
                            const int nlx = lx + dx;
                            const int nly = ly + dy;
                            if (nlx < 0 || nlx >= tw || nly < 0 || nly >= th) {
                                touches_seam = 1;
                                continue;
                            }
                            const int q = nly * tw + nlx;
                            if (!visited[q]) {
                                visited[q] = 1;
                                queue[tail++] = q;
                            }
                        }
                    }
                }
                fragments += touches_seam;
            }
            counts[ty * tiles_x + tx] = (uint16_t)fragments;
        }
    }
    free(visited);
    free(queue);
    return 0;
}

int ss_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

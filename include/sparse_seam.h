/*
 * sparse_seam.h -- C ABI of the B200-native exact dual regional-extrema route.
 *
 * Given an 8-bit grayscale image, the library writes two byte masks:
 *   maxima[y][x] = 255 iff the 8-connected equal-valued flat zone of (x, y)
 *                  has no strictly greater 8-neighbour, else 0;
 *   minima[y][x] = 255 iff it has no strictly smaller 8-neighbour, else 0.
 * Pixels outside the image are absent.  The masks are bit-exact against the
 * reference's Sparse-Seam and Global-UF routes and against MATLAB
 * imregionalmax / imregionalmin(img, 8).
 *
 * Everything crosses this boundary as plain pointers and sizes.  Device
 * pointers are CUDA global-memory addresses of the current device; `stream`
 * is a cudaStream_t passed as void* (NULL = the legacy default stream).
 * No function throws.  The device entry points only enqueue work on the
 * stream: they allocate nothing, never synchronise and may be captured into a
 * CUDA graph.  One workspace serves one call in flight at a time; distinct
 * workspaces on distinct streams may run concurrently from any host threads.
 *
 * Reference interfaces replaced (paths inside the reference repository):
 *   ss_workspace_bytes   <- allocate_buffers sizing
 *                           (harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:710-737)
 *                           and memory accounting
 *                           (harness/primary/gpu_common_v0_6.cu:410-429)
 *   ss_workspace_init    <- per-run cudaMemset of error_flag
 *                           (harness/primary/gpu_common_v0_6.cu:147)
 *   ss_extrema           <- run_sparse_resident
 *                           (harness/primary/gpu_common_v0_6.cu:137-206)
 *   ss_read_status       <- error_flag and tile_fragment_counts read-back
 *                           (harness/primary/gpu_common_v0_6.cu:377-387,
 *                            snapshot_sparse_seam_cuda_v1_0.cu:840-863)
 *   ss_extrema_host      <- run_sparse_seam: H2D, kernels, D2H, kernel ms,
 *                           active fragments
 *                           (harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:753-878)
 *   ss_batch_*           <- the per-image host loop of the harness
 *                           (harness/primary/gpu_common_v0_6.cu:584-745),
 *                           replaced by one launch over many images.
 */
#ifndef SPARSE_SEAM_H
#define SPARSE_SEAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SS_ABI_VERSION 2

typedef enum ss_status {
    SS_OK = 0,
    /* Host-side argument checks (nothing was enqueued). */
    SS_ERR_INVALID_VALUE = 1,      /* NULL pointer, non-positive size, pitch < width */
    SS_ERR_UNSUPPORTED_TILE = 2,   /* tile not in {16, 32, 64} */
    SS_ERR_WORKSPACE_TOO_SMALL = 3,
    SS_ERR_MISALIGNED = 4,         /* workspace / plan not 256-byte aligned */
    SS_ERR_TOO_LARGE = 5,          /* beyond 32-bit pixel or fragment indexing */
    SS_ERR_CUDA = 6,               /* a CUDA runtime call failed */
    /* Device-side invariants, reported by ss_read_status. */
    SS_ERR_FRAGMENT_OVERFLOW = 7,  /* a tile produced more seam fragments than
                                      its slots (reference error_flag 1) */
    SS_ERR_RECORD_RANGE = 8,       /* a fragment record out of range
                                      (reference error_flag 2) */
    SS_ERR_INVARIANT = 9,          /* a union-find link broke the min-root
                                      order or left the arena (reference
                                      error_flag 3) */
    SS_ERR_SPIN_LIMIT = 10,        /* a bounded device loop gave up */
    SS_ERR_WORKSPACE_UNINITIALIZED = 11, /* ss_workspace_init was not run */
    SS_ERR_HOST_ALLOC = 12,        /* host-side allocation failed */
    SS_ERR_EXCEEDS_STATIC_SCRATCH = 13 /* the image needs more scratch than
                                          ss_extrema_static_scratch holds */
} ss_status;

/* Human-readable name of a status code (static storage). */
const char* ss_status_string(ss_status status);

/* ABI version of the loaded library (SS_ABI_VERSION). */
int ss_abi_version(void);

/* Bytes of device workspace one call needs for a width x height image with
 * the given tile size (16, 32 or 64).  The workspace holds the seam-fragment
 * union-find arena (4*tile slots per tile), the per-tile border records, the
 * per-tile fragment counts and seam-pair counters, and a status header. */
ss_status ss_workspace_bytes(int width, int height, int tile, size_t* bytes);

/* Resets a workspace (status header and seam-pair counters).  Required once
 * after allocation, and again after any call whose status was not SS_OK. */
ss_status ss_workspace_init(void* d_workspace, size_t workspace_bytes,
                            void* stream);

/* Enqueues the route for one device-resident image.
 *   d_image    width x height bytes, rows `pitch` bytes apart (pitch >= width)
 *   d_maxima,
 *   d_minima   outputs, rows `out_pitch` bytes apart; 0/255 bytes
 *   tile       16, 32 or 64: seam-fragment tile edge (the reference's SS_TILE)
 * The masks do not depend on `tile`; only speed and the fragment statistics
 * do.  Device-side invariant failures are recorded in the workspace header
 * and returned by ss_read_status. */
ss_status ss_extrema(const uint8_t* d_image, int width, int height, int pitch,
                     int tile, uint8_t* d_maxima, uint8_t* d_minima,
                     int out_pitch, void* d_workspace, size_t workspace_bytes,
                     void* stream);

typedef struct ss_stats {
    uint32_t device_error;        /* ss_status of the first device invariant
                                     failure since the last read, or 0 */
    uint32_t error_detail;        /* implementation detail of that failure */
    uint64_t active_fragments;    /* seam fragments of the last call (sum
                                     of per-tile counts).  The CTA-per-tile
                                     kernels create one per seam-touching
                                     tile-local zone, exactly the reference's
                                     tile_fragment_counts; the row-scan
                                     kernels only one per seam zone whose
                                     verdict the merge can still change */
    uint64_t tiles;               /* tiles of the last call */
    uint64_t flipped_tiles;       /* tiles whose seam fragments changed
                                     verdict after the global merge */
    uint64_t live_pixels;         /* pixels whose verdict waited for the
                                     global merge (the runs of live seam
                                     zones; row-scan kernels only, else 0):
                                     the seam-pixel share is this over the
                                     call's pixels */
} ss_stats;

/* Kernel configuration used for a tile size by every later call of this
 * process (the autotuner's hook; the masks never depend on it).
 *   warps > 0   CTA-per-tile kernels with `warps` warps per CTA
 *               (tile 16: 2, 4 or 8; tile 32: 4, 8 or 16; tile 64: 8 or 16)
 *   warps < 0   row-scan kernels (per-row bit masks and runs): tile 32, one
 *               tile per warp, -warps warps per CTA (2 or 4); tile 64 (-4),
 *               one tile per CTA of four warps, one per 32 x 32 quadrant
 * Defaults: tile 16 -> 4, tile 32 -> -4, tile 64 -> -4.  The reference fixes
 * its tile and classify threads at compile time
 * (harness/configuration_study/sparse_config_benchmark_v0_8.cu:17-30). */
ss_status ss_set_kernel_config(int tile, int warps);
ss_status ss_get_kernel_config(int tile, int* warps);

/* Measurement aid: enqueues `count` launches of an empty kernel with `grid`
 * CTAs of `threads` threads on `stream`.  Replayed from a CUDA graph with the
 * grid shapes of a route call, it gives the launch floor that no launch-based
 * route can go below.  No counterpart in the reference. */
ss_status ss_empty_launches(int count, int grid, int threads, void* stream);

/* Zero-allocation form of ss_extrema, for callers that cannot allocate
 * device memory (code that must not enter the allocator: another
 * allocator's callback, a latency-critical loop, a plug-in whose host owns
 * every device allocation).  No counterpart in the reference, which always
 * allocates per image.  The route's scratch is a fixed 32 MiB array inside
 * the library; this call allocates nothing (no cudaMalloc, no allocating
 * library routine).
 * Limits: images whose ss_workspace_bytes exceeds 32 MiB are rejected with
 * SS_ERR_EXCEEDS_STATIC_SCRATCH (at T = 32 about 4.8 Mpixel, e.g. 2040 x 1356
 * or 2208 x 2208; at T = 64 about 5.9 Mpixel; at T = 16 about 14 Mpixel).
 * Set-up: the array lives in its own module, which the driver loads (and so
 * allocates the 32 MiB) the first time this call or
 * ss_static_scratch_read_status runs in a CUDA context; the first call in a
 * context also clears the array and waits for the clear on `stream`.  So make
 * a first call (a warm-up) outside the no-allocation context and before any
 * stream capture.  The array is then held on that GPU until the process
 * exits.
 * Every call shares the one array and it keeps the previous call's contents,
 * so each call clears what must start at zero (including the error word);
 * calls that overlap on the GPU (other streams, other host threads) race and
 * must be serialised by the caller.  Device-side invariant failures of a call
 * are read with ss_static_scratch_read_status before the next call. */
ss_status ss_extrema_static_scratch(const uint8_t* d_image, int width,
                                    int height, int pitch, int tile,
                                    uint8_t* d_maxima, uint8_t* d_minima,
                                    int out_pitch, void* stream);

/* Synchronises `stream`, copies the status header (and, if `stats` is not
 * NULL, the statistics) to the host and clears the device error word.
 * Returns SS_OK or the first device-side failure. */
ss_status ss_read_status(void* d_workspace, size_t workspace_bytes,
                         void* stream, ss_stats* stats);

/* ss_read_status for the array of ss_extrema_static_scratch in the current
 * context: synchronises `stream` and returns SS_OK or the device-side
 * failure of the last call (SS_ERR_WORKSPACE_UNINITIALIZED if no call has
 * set the array up in this context).  Allocates no device memory.  No
 * counterpart in the reference. */
ss_status ss_static_scratch_read_status(void* stream, ss_stats* stats);

/* Host-to-host convenience form: copies a host image to the device, runs
 * ss_extrema, copies both masks back and synchronises.  Device buffers are
 * owned by an opaque context, so repeated calls reuse them.
 * `elapsed_ms` (optional) receives the device time of the kernels alone;
 * `active_fragments` (optional) the fragment count. */
typedef struct ss_context ss_context;
ss_status ss_context_create(int device, ss_context** context);
void ss_context_destroy(ss_context* context);
ss_status ss_extrema_host(ss_context* context, const uint8_t* h_image,
                          int width, int height, int pitch, int tile,
                          uint8_t* h_maxima, uint8_t* h_minima, int out_pitch,
                          float* elapsed_ms, uint64_t* active_fragments);

/* ---------------------------------------------------------------------- */
/* Batches: many images of uneven sizes in one launch pair.                */
/* ---------------------------------------------------------------------- */

typedef struct ss_image_desc {
    const uint8_t* image;   /* device pointer */
    uint8_t* maxima;        /* device pointer */
    uint8_t* minima;        /* device pointer */
    int32_t width;
    int32_t height;
    int32_t pitch;
    int32_t out_pitch;
} ss_image_desc;

/* Size of the device plan for `count` images and `total_tiles` tiles (the
 * sum over images of ceil(w/tile)*ceil(h/tile); pass 0 to have it computed
 * by ss_batch_plan_fill). */
ss_status ss_batch_plan_bytes(int count, int64_t total_tiles, size_t* bytes);

/* Counts the tiles of a batch for a given tile size. */
ss_status ss_batch_tiles(const ss_image_desc* descs, int count, int tile,
                         int64_t* total_tiles);

/* Fills a HOST buffer with the plan (image table, tile offsets and the
 * tile-to-image map) for `descs`.  The caller copies it to a 256-byte aligned
 * device buffer of the same size (e.g. cudaMemcpyAsync) before
 * ss_extrema_batch; a plan stays valid for as long as the images' pointers
 * and sizes do, so it can be reused across calls and graph replays.
 * `workspace_bytes` (optional) receives the workspace size the batch needs. */
ss_status ss_batch_plan_fill(const ss_image_desc* descs, int count, int tile,
                             void* h_plan, size_t plan_bytes,
                             size_t* workspace_bytes);

/* Enqueues the route over every image of a plan.  `h_plan` is the host plan
 * filled by ss_batch_plan_fill (read for sizes, and for the image entry of
 * a one-image plan, which travels in the launch parameters), `d_plan` its
 * device copy (read by the kernels); the two must hold the same bytes when
 * the call is made (or captured).  Each image gets its own seam-fragment arena
 * inside the workspace; results are the same as calling ss_extrema on each
 * image alone.
 *   persistent  0: one CTA per (image, tile) work item;
 *               1: a persistent grid (one wave of CTAs) that pops
 *                  (image, tile) items from a device work queue. */
ss_status ss_extrema_batch(const void* h_plan, const void* d_plan,
                           size_t plan_bytes, int persistent,
                           void* d_workspace, size_t workspace_bytes,
                           void* stream);

/* Split form of ss_extrema_batch: pass 1 is the tile pass, pass 4 the seam
 * pass (row-scan kernels only; a no-op for the others), pass 2 the resolve
 * pass.  Enqueuing passes 1, 4 and 2 in that order on one stream (other work
 * may sit between them, e.g. timing events) is exactly ss_extrema_batch; the
 * `persistent` flag must be the same for all passes. */
ss_status ss_extrema_batch_pass(const void* h_plan, const void* d_plan,
                                size_t plan_bytes, int persistent, int pass,
                                void* d_workspace, size_t workspace_bytes,
                                void* stream);

/* Re-quantisation fused into the tile load: the masks are those of the image
 * re-quantised to `levels` gray levels (2..256) with the reference's rule
 * bin = (v * levels) >> 8, v' = (bin * 255 + (levels - 1) / 2) / (levels - 1)
 * (harness/quantization_and_scaling/gpu_common_quant_v0_7.cu:479-494, where
 * it runs on the host before the copy); the image itself is not changed.
 * levels 0 or 256: the image as it is.  ss_extrema_levels is ss_extrema with
 * that option; ss_batch_plan_set_levels sets it for image `index` of a host
 * plan (before the plan is copied to the device). */
ss_status ss_extrema_levels(const uint8_t* d_image, int width, int height,
                            int pitch, int tile, int levels,
                            uint8_t* d_maxima, uint8_t* d_minima,
                            int out_pitch, void* d_workspace,
                            size_t workspace_bytes, void* stream);
ss_status ss_batch_plan_set_levels(void* h_plan, size_t plan_bytes, int index,
                                   int levels);

/* Per-call launch choices: the knobs of the batch autotuner.  None of them
 * changes the masks.  No counterpart in the reference, whose tile, classify
 * threads and flatten launch are compile-time constants
 * (harness/configuration_study/sparse_config_benchmark_v0_8.cu:17-30). */
typedef struct ss_launch {
    int32_t warps;       /* kernel family for the plan's tile, as in
                          * ss_set_kernel_config; 0 = the tile's current
                          * default */
    int32_t persistent;  /* 0 grid schedule, 1 persistent work queue */
    int32_t group;       /* row-scan seam and resolve passes: tiles per warp,
                          * 1, 2, 4, 8, 16 or 32; 0 = chosen from the tile
                          * count (one tile per warp for small launches, up to
                          * 32 for large ones) */
    int32_t passes;      /* passes to enqueue (1 tile, 4 seam, 2 resolve,
                          * enqueued in that order); 0 = all */
    int32_t flatten;     /* row-scan kernels: flatten schedule of the seam
                          * fragments' union-find before the verdicts are
                          * read.  0 = roots found with path halving in the
                          * flags pass; 1 = also point every fragment at its
                          * root there; 2 = a separate pass points every
                          * fragment at its root first (the reference's
                          * compress_fragment_parents,
                          * harness/primary/snapshot_sparse_seam_cuda_v1_0.cu
                          * :583-599), one more launch */
} ss_launch;

/* ss_extrema_batch with explicit launch choices (NULL = all defaults). */
ss_status ss_extrema_batch_launch(const void* h_plan, const void* d_plan,
                                  size_t plan_bytes, const ss_launch* launch,
                                  void* d_workspace, size_t workspace_bytes,
                                  void* stream);

/* ---------------------------------------------------------------------- */
/* Compact host-to-host transfer of the masks.                              */
/* ---------------------------------------------------------------------- */
/* Host-to-host throughput is bound by the bus: 1 byte per pixel goes in and
 * two mask bytes come back.  ss_pack_masks packs `n` consecutive mask bytes
 * of each mask (any non-zero byte = 1) into bit planes on the device, bit i
 * of word i / 32 for pixel i, (n + 31) / 32 words each; after the planes are
 * copied to the host, ss_unpack_masks writes the 0/255 bytes into the host
 * masks with `threads` host threads (0 = all processors but one), and
 * ss_enqueue_unpack_masks
 * does the same as a host function enqueued on `stream` (ordered after the
 * stream's earlier work; the buffers must stay valid until it runs; 0 = a
 * quarter of the processors, at least one: the expansion then overlaps
 * host-to-device copies that read the same host memory, and more threads
 * slow those copies more than they speed the expansion).  No
 * counterpart in the reference, which copies both byte masks back
 * (harness/primary/gpu_common_v0_6.cu:351-373). */
ss_status ss_pack_masks(const uint8_t* d_maxima, const uint8_t* d_minima,
                        uint64_t n, uint32_t* d_max_bits,
                        uint32_t* d_min_bits, void* stream);
ss_status ss_unpack_masks(const uint32_t* h_max_bits,
                          const uint32_t* h_min_bits, uint64_t n,
                          uint8_t* h_maxima, uint8_t* h_minima, int threads);
ss_status ss_enqueue_unpack_masks(const uint32_t* h_max_bits,
                                  const uint32_t* h_min_bits, uint64_t n,
                                  uint8_t* h_maxima, uint8_t* h_minima,
                                  int threads, void* stream);

/* ---------------------------------------------------------------------- */
/* Image files.                                                            */
/* ---------------------------------------------------------------------- */
/* Reads a PGM (P5 / P2, maxval <= 255), PNG (any colour type, 1/2/4/8-bit
 * samples, not interlaced), BMP (1/4/8-bit palettes, 16/24/32-bit, RLE8 /
 * RLE4), JPEG (sequential or progressive Huffman, 8-bit, gray or YCbCr; EXIF orientation
 * applied) or TIFF (strips / tiles, none / LZW / Deflate / PackBits, 1/8/16-
 * bit gray, 8-bit RGB(A) and palette) as 8-bit gray, as the reference's
 * cv::imread(path, IMREAD_GRAYSCALE) does
 * (harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:87-103).  With `pixels`
 * NULL only `width` and `height` are filled; otherwise `capacity` must hold
 * width * height bytes (rows packed).  SS_ERR_INVALID_VALUE for an unreadable
 * or unsupported file. */
ss_status ss_read_image(const char* path, uint8_t* pixels, size_t capacity,
                        int* width, int* height);
/* Writes a binary PGM (P5, maxval 255). */
ss_status ss_write_pgm(const char* path, const uint8_t* pixels, int width,
                       int height, int pitch);

/* ---------------------------------------------------------------------- */
/* Serving: a continuous-batching request loop on one GPU.                 */
/* ---------------------------------------------------------------------- */
/* No counterpart in the reference, whose harness runs one image at a time
 * (harness/primary/gpu_common_v0_6.cu:137-206).  A server owns, for its
 * lifetime, a device pool for request buffers and `inflight` batch slots
 * (a stream, a DSU workspace for `batch_tiles` tiles and a plan buffer
 * each).  A worker thread admits submitted requests in arrival order as pool
 * memory frees up (admission by HBM footprint: image plus two masks), copies
 * their images in on a copy stream, and whenever a slot is free launches
 * every admitted request not yet launched as one batch (ss_extrema_batch),
 * so requests arriving while others run join the next batch and batches
 * overlap on the device.  Each slot's stream then copies the masks out,
 * reads the batch's device status and frees the requests' pool memory.
 * Masks are the same as ss_extrema's on each image alone.  Thread-safe:
 * any thread may submit and poll. */

#define SS_REQUEST_DEVICE 1u  /* image and masks are device pointers owned by
                               * the caller: no pool memory, no copies */

typedef struct ss_request {
    const uint8_t* image;   /* host (pinned for overlap) or device pointer */
    uint8_t* maxima;
    uint8_t* minima;
    int32_t width;
    int32_t height;
    int32_t pitch;
    int32_t out_pitch;
    uint32_t flags;         /* SS_REQUEST_* */
    uint32_t reserved;
    uint64_t user;          /* returned in the completion */
} ss_request;

typedef struct ss_completion {
    uint64_t ticket;
    uint64_t user;
    int32_t status;         /* SS_OK or the batch's device failure */
    int32_t batch_images;   /* requests in the batch that carried it */
    int64_t submit_ns;      /* CLOCK_MONOTONIC nanoseconds */
    int64_t admit_ns;       /* pool memory granted, copy-in enqueued */
    int64_t launch_ns;      /* batch enqueued */
    int64_t done_ns;        /* masks in the caller's buffers */
} ss_completion;

typedef struct ss_server_config {
    int32_t device;           /* CUDA device ordinal */
    int32_t tile;             /* 16, 32 or 64 */
    int32_t persistent;       /* batch schedule, as in ss_extrema_batch */
    int32_t inflight;         /* batch slots, 1..16 */
    int32_t max_batch_images; /* requests per batch, >= 1 */
    int32_t unpack_threads;   /* host masks of 8 Mpixel or more with
                               * out_pitch == width come back as bit planes
                               * (ss_pack_masks) expanded by this many host
                               * threads (0: half the host's processors);
                               * -1: byte copies of every mask */
    int64_t batch_tiles;      /* tile capacity of one batch's workspace */
    uint64_t pool_bytes;      /* device bytes for request images and masks */
} ss_server_config;

typedef struct ss_server_stats {
    uint64_t submitted;
    uint64_t completed;
    uint64_t batches;
    uint64_t pixels;               /* of completed requests */
    uint64_t pool_bytes;
    uint64_t pool_high_water;      /* most pool bytes in use at once */
    uint32_t max_batch_images_seen;
    uint32_t inflight_high_water;  /* most batches on the device at once */
} ss_server_stats;

typedef struct ss_server ss_server;

/* Allocates the pool and slots on `config->device` and starts the worker.
 * Fails with SS_ERR_INVALID_VALUE / SS_ERR_UNSUPPORTED_TILE on a bad config
 * (checked before any CUDA call), SS_ERR_TOO_LARGE if `batch_tiles` exceeds
 * the workspace's index range, SS_ERR_CUDA on allocation failure. */
ss_status ss_server_create(const ss_server_config* config,
                           ss_server** server);

/* Queues one request; `ticket` (optional) receives its id.  Rejected at once
 * with SS_ERR_TOO_LARGE if it can never fit (more tiles than batch_tiles or
 * more bytes than the pool), SS_ERR_INVALID_VALUE on bad geometry. */
ss_status ss_server_submit(ss_server* server, const ss_request* request,
                           uint64_t* ticket);

/* Moves up to `capacity` completions into `out`, waiting up to `timeout_us`
 * microseconds for the first one (0: no wait).  `count` receives how many. */
ss_status ss_server_poll(ss_server* server, ss_completion* out, int capacity,
                         int* count, int timeout_us);

ss_status ss_server_get_stats(ss_server* server, ss_server_stats* stats);

/* Finishes every submitted request, stops the worker and frees the server's
 * memory.  Completions not yet polled are dropped. */
void ss_server_destroy(ss_server* server);

#ifdef __cplusplus
}
#endif

#endif /* SPARSE_SEAM_H */

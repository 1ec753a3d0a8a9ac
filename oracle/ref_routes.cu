// ref_routes.cu -- C entry points around the reference's own GPU routes.
//
// CHECKER ONLY (test infrastructure).  This translation unit textually
// includes the reference's unified harness, harness/primary/gpu_common_v0_6.cu,
// from the reference tree at build time (oracle/ref_build.py passes its
// directory with -I), exactly as that harness includes the Sparse-Seam v1.0
// and Global-UF snapshots.  Nothing of the reference is copied here; the
// functions below only call the reference's own benchmark routines
// (benchmark_sparse_v02, gpu_common_v0_6.cu:305-399; benchmark_common_v02 with
// run_global_uf, gpu_common_v0_6.cu:211-303 and
// snapshot_gpu_benchmark_globaluf_ole_v0_1.cu:341-385) so that the parity
// tests can compare the product's masks with the reference's routes compiled
// for sm_100a, and the benchmark can time them beside the product.
#include "gpu_common_v0_6.cu"

#include <cstdint>
#include <cstring>
#include <exception>

namespace {

cv::Mat wrap_copy(const std::uint8_t* image, int width, int height) {
    cv::Mat m;
    m.create(height, width, CV_8U);
    std::memcpy(m.data, image, static_cast<size_t>(width) * height);
    return m;
}

}  // namespace

extern "C" int ssref_tile(void) { return TILE; }

// Sparse-Seam v1.0 through the reference harness's resident benchmark.
// Returns 0, or -1 if the reference route threw (CUDA error or its device
// invariant flag).
extern "C" int ssref_sparse_seam(const std::uint8_t* image, int width,
                                 int height, std::uint8_t* maxima,
                                 std::uint8_t* minima, int warmup, int reps,
                                 double* median_ms, double* median_h2h_ms,
                                 long long* active_fragments) {
    try {
        const int pixels = width * height;
        const int tiles_x = (width + TILE - 1) / TILE;
        const int tiles_y = (height + TILE - 1) / TILE;
        const int tiles = tiles_x * tiles_y;
        SparseDeviceBuffers buffers;
        sparse_allocate_buffers(buffers, pixels, tiles * SLOTS_PER_TILE);
        cv::Mat img = wrap_copy(image, width, height);
        cv::Mat mx;
        cv::Mat mn;
        const unified_v05::Timing t = unified_v05::benchmark_sparse_v02(
            buffers, img, warmup, reps, mx, mn);
        std::vector<std::uint16_t> counts(static_cast<size_t>(tiles));
        CUDA_CHECK_V2(cudaMemcpy(counts.data(), buffers.tile_fragment_counts,
                                 counts.size() * sizeof(std::uint16_t),
                                 cudaMemcpyDeviceToHost));
        long long sum = 0;
        for (std::uint16_t c : counts) {
            sum += c;
        }
        sparse_free_buffers(buffers);
        std::memcpy(maxima, mx.data, static_cast<size_t>(pixels));
        std::memcpy(minima, mn.data, static_cast<size_t>(pixels));
        if (median_ms) *median_ms = t.median_compute_ms;
        if (median_h2h_ms) *median_h2h_ms = t.median_h2h_ms;
        if (active_fragments) *active_fragments = sum;
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// Global-UF through the reference harness's common benchmark.
extern "C" int ssref_global_uf(const std::uint8_t* image, int width,
                               int height, std::uint8_t* maxima,
                               std::uint8_t* minima, int warmup, int reps,
                               double* median_ms, double* median_h2h_ms) {
    try {
        const int pixels = width * height;
        CommonDeviceBuffers buffers;
        common_allocate_buffers(buffers, pixels);
        cv::Mat img = wrap_copy(image, width, height);
        cv::Mat mx;
        cv::Mat mn;
        const unified_v05::Timing t = unified_v05::benchmark_common_v02(
            run_global_uf, buffers, img, 16, warmup, reps, mx, mn);
        common_free_buffers(buffers);
        std::memcpy(maxima, mx.data, static_cast<size_t>(pixels));
        std::memcpy(minima, mn.data, static_cast<size_t>(pixels));
        if (median_ms) *median_ms = t.median_compute_ms;
        if (median_h2h_ms) *median_h2h_ms = t.median_h2h_ms;
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

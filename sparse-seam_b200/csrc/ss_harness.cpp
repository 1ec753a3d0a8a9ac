// ss_harness.cpp -- command-line benchmark harness over the C ABI.
//
// Same command line, CSV columns and environment file as the reference's
// harness (harness/primary/gpu_common_v0_6.cu:479-640), with the Sparse-Seam
// route replaced by this library:
//
//   ss_harness <image_dir> --output=DIR [--expected-max=DIR --expected-min=DIR]
//              [--device=0] [--block=16] [--warmup=5] [--reps=30]
//              [--tile=32] [--masks]
//
// For every .pgm / .png / .bmp / .jpg / .jpeg / .tif / .tiff file of
// <image_dir> (sorted by name): the image is
// read as 8-bit gray, copied to the device once, run `warmup` times, then
// `reps` times timed with CUDA events (compute: device-resident input) and
// `reps` times timed on the host clock from the host image to both host
// masks (h2h: copy in, route, copy both masks out).  Masks are compared with
// the expected masks of the same file name (PGM, PNG or BMP), if given
// ("oracle" columns), and with a second, independent kernel family of this
// library (CTA-per-tile kernels at the same tile; "cross" columns).  The
// row's memory columns count this route's device buffers: the image, both
// masks and the workspace ("auxiliary" = the workspace).  `--block` is read
// and recorded for command-line compatibility.  `--masks` also writes the
// masks as PGM files into DIR/masks.  Exit status 0 when every comparison
// matched, 1 on a mismatch, 2 on a usage error, 3 on any other failure.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "sparse_seam.h"
#include "ss_percentile.hpp"

namespace fs = std::filesystem;

namespace {

struct Timing {
    double median_compute_ms = 0, p95_compute_ms = 0;
    double median_h2h_ms = 0, p95_h2h_ms = 0;
};

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string(what) + ": " +
                                 cudaGetErrorString(e));
    }
}

void check_ss(ss_status s, const char* what) {
    if (s != SS_OK) {
        throw std::runtime_error(std::string(what) + ": " +
                                 ss_status_string(s));
    }
}

using ss_harness::percentile;

std::string quote(const std::string& s) {
    std::string out = "\"";
    for (char c : s) {
        if (c == '"') out += '"';
        out += c;
    }
    return out + "\"";
}

std::vector<uint8_t> read_image(const fs::path& p, int& w, int& h) {
    check_ss(ss_read_image(p.string().c_str(), nullptr, 0, &w, &h),
             ("cannot read " + p.string()).c_str());
    std::vector<uint8_t> px(static_cast<size_t>(w) * h);
    check_ss(ss_read_image(p.string().c_str(), px.data(), px.size(), &w, &h),
             ("cannot read " + p.string()).c_str());
    return px;
}

// Expected mask of `stem` in `dir` (.pgm, else .png, else .bmp, else .tif), or
// an empty vector.
std::vector<uint8_t> expected(const fs::path& dir, const std::string& stem,
                              int w, int h) {
    for (const char* ext : {".pgm", ".png", ".bmp", ".tif"}) {
        const fs::path p = dir / (stem + ext);
        if (fs::exists(p)) {
            int ew = 0, eh = 0;
            std::vector<uint8_t> m = read_image(p, ew, eh);
            if (ew != w || eh != h) {
                throw std::runtime_error("expected mask size differs: " +
                                         p.string());
            }
            return m;
        }
    }
    return {};
}

uint64_t mismatches(const std::vector<uint8_t>& a,
                    const std::vector<uint8_t>& b) {
    uint64_t n = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        n += (a[i] != 0) != (b[i] != 0);
    }
    return n;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "Usage: ss_harness <image_dir> --output=DIR"
                     " [--expected-max=DIR --expected-min=DIR]"
                     " [--device=0] [--block=16] [--warmup=5] [--reps=30]"
                     " [--tile=32] [--masks]\n";
        return 2;
    }
    try {
        const fs::path image_dir = argv[1];
        fs::path output_dir, expected_max_dir, expected_min_dir;
        int device = 0, block = 16, warmup = 5, reps = 30, tile = 32;
        bool save_masks = false;
        for (int i = 2; i < argc; ++i) {
            const std::string a = argv[i];
            auto value = [&](const char* key) -> const char* {
                const size_t n = std::strlen(key);
                return a.compare(0, n, key) == 0 ? a.c_str() + n : nullptr;
            };
            if (const char* v = value("--output=")) output_dir = v;
            else if (const char* v = value("--expected-max=")) expected_max_dir = v;
            else if (const char* v = value("--expected-min=")) expected_min_dir = v;
            else if (const char* v = value("--device=")) device = std::stoi(v);
            else if (const char* v = value("--block=")) block = std::stoi(v);
            else if (const char* v = value("--warmup=")) warmup = std::stoi(v);
            else if (const char* v = value("--reps=")) reps = std::stoi(v);
            else if (const char* v = value("--tile=")) tile = std::stoi(v);
            else if (a == "--masks") save_masks = true;
            else {
                std::cerr << "unknown option " << a << "\n";
                return 2;
            }
        }
        if (output_dir.empty()) {
            std::cerr << "Missing --output directory\n";
            return 2;
        }
        if (expected_max_dir.empty() != expected_min_dir.empty()) {
            std::cerr << "Expected max/min directories must be supplied "
                         "together\n";
            return 2;
        }
        if (warmup < 0 || reps < 1 || (tile != 16 && tile != 32 && tile != 64)) {
            std::cerr << "Invalid benchmark option\n";
            return 2;
        }
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        cudaDeviceProp prop{};
        check_cuda(cudaGetDeviceProperties(&prop, device),
                   "cudaGetDeviceProperties");
        fs::create_directories(output_dir);
        if (save_masks) fs::create_directories(output_dir / "masks");
        std::ofstream csv(output_dir / "ss_harness.csv");
        if (!csv) throw std::runtime_error("cannot create the CSV");
        csv << "algorithm,image,width,height,megapixels,warmup,repetitions,"
               "block,total_allocated_bytes,total_allocated_Bpp,"
               "auxiliary_bytes,auxiliary_Bpp,"
               "median_compute_ms,p95_compute_ms,compute_mpix_s,"
               "median_h2h_ms,p95_h2h_ms,h2h_mpix_s,"
               "median_iterations,p95_iterations,"
               "oracle_max_mismatches,oracle_min_mismatches,"
               "cross_max_mismatches,cross_min_mismatches\n";
        int kernel = 0;
        ss_get_kernel_config(tile, &kernel);
        {
            std::ofstream env(output_dir / "environment.txt");
            env << "harness=ss_harness\n"
                << "device_name=" << prop.name << '\n'
                << "compute_capability=" << prop.major << '.' << prop.minor
                << '\n'
                << "global_memory_bytes=" << prop.totalGlobalMem << '\n'
                << "cuda_runtime=" << CUDART_VERSION << '\n'
                << "abi_version=" << ss_abi_version() << '\n'
                << "block=" << block << '\n'
                << "warmup=" << warmup << '\n'
                << "repetitions=" << reps << '\n'
                << "tile=" << tile << '\n'
                << "kernel_config=" << kernel << '\n'
                << "timing_compute=preallocated,resident_input,task_complete\n"
                << "timing_h2h=reused_allocation,H2D+compute+D2H_two_masks\n"
                << "auxiliary_definition=all_device_buffers_except_input_and_"
                   "two_output_masks\n";
        }

        std::vector<fs::path> files;
        for (const auto& e : fs::directory_iterator(image_dir)) {
            const std::string ext = e.path().extension().string();
            if (e.is_regular_file() &&
                (ext == ".pgm" || ext == ".png" || ext == ".bmp" ||
                 ext == ".jpg" || ext == ".jpeg" || ext == ".tif" ||
                 ext == ".tiff")) {
                files.push_back(e.path());
            }
        }
        std::sort(files.begin(), files.end());
        uint64_t total_oracle = 0, total_cross = 0;
        cudaStream_t stream = nullptr;
        check_cuda(cudaStreamCreate(&stream), "cudaStreamCreate");
        cudaEvent_t ev0, ev1;
        check_cuda(cudaEventCreate(&ev0), "cudaEventCreate");
        check_cuda(cudaEventCreate(&ev1), "cudaEventCreate");
        for (const fs::path& path : files) {
            int w = 0, h = 0;
            std::vector<uint8_t> img = read_image(path, w, h);
            const size_t n = img.size();
            size_t ws_bytes = 0;
            check_ss(ss_workspace_bytes(w, h, tile, &ws_bytes),
                     "ss_workspace_bytes");
            uint8_t *d_img = nullptr, *d_max = nullptr, *d_min = nullptr;
            void* d_ws = nullptr;
            check_cuda(cudaMalloc(&d_img, n), "cudaMalloc");
            check_cuda(cudaMalloc(&d_max, n), "cudaMalloc");
            check_cuda(cudaMalloc(&d_min, n), "cudaMalloc");
            check_cuda(cudaMalloc(&d_ws, ws_bytes), "cudaMalloc");
            check_ss(ss_workspace_init(d_ws, ws_bytes, stream),
                     "ss_workspace_init");
            uint8_t *h_img = nullptr, *h_max = nullptr, *h_min = nullptr;
            check_cuda(cudaMallocHost(&h_img, n), "cudaMallocHost");
            check_cuda(cudaMallocHost(&h_max, n), "cudaMallocHost");
            check_cuda(cudaMallocHost(&h_min, n), "cudaMallocHost");
            std::memcpy(h_img, img.data(), n);
            auto route = [&] {
                check_ss(ss_extrema(d_img, w, h, w, tile, d_max, d_min, w,
                                    d_ws, ws_bytes, stream),
                         "ss_extrema");
            };
            check_cuda(cudaMemcpyAsync(d_img, h_img, n, cudaMemcpyHostToDevice,
                                       stream), "H2D");
            for (int i = 0; i < warmup; ++i) route();
            check_cuda(cudaStreamSynchronize(stream), "warm-up");
            Timing t;
            std::vector<double> compute, h2h;
            for (int r = 0; r < reps; ++r) {
                check_cuda(cudaEventRecord(ev0, stream), "event");
                route();
                check_cuda(cudaEventRecord(ev1, stream), "event");
                check_cuda(cudaEventSynchronize(ev1), "event");
                float ms = 0;
                check_cuda(cudaEventElapsedTime(&ms, ev0, ev1), "event");
                compute.push_back(ms);
            }
            for (int r = 0; r < reps; ++r) {
                const auto b = std::chrono::high_resolution_clock::now();
                check_cuda(cudaMemcpyAsync(d_img, h_img, n,
                                           cudaMemcpyHostToDevice, stream),
                           "H2D");
                route();
                check_cuda(cudaMemcpyAsync(h_max, d_max, n,
                                           cudaMemcpyDeviceToHost, stream),
                           "D2H");
                check_cuda(cudaMemcpyAsync(h_min, d_min, n,
                                           cudaMemcpyDeviceToHost, stream),
                           "D2H");
                check_cuda(cudaStreamSynchronize(stream), "h2h");
                const auto e = std::chrono::high_resolution_clock::now();
                h2h.push_back(
                    std::chrono::duration<double, std::milli>(e - b).count());
            }
            ss_stats stats{};
            check_ss(ss_read_status(d_ws, ws_bytes, stream, &stats),
                     ("device status of " + path.string()).c_str());
            t.median_compute_ms = percentile(compute, 0.5);
            t.p95_compute_ms = percentile(compute, 0.95);
            t.median_h2h_ms = percentile(h2h, 0.5);
            t.p95_h2h_ms = percentile(h2h, 0.95);
            std::vector<uint8_t> mx(h_max, h_max + n), mn(h_min, h_min + n);

            // Cross route: the CTA-per-tile kernels of the same tile.
            uint64_t cross_max = 0, cross_min = 0;
            {
                int saved = 0;
                ss_get_kernel_config(tile, &saved);
                const int other = tile == 16 ? 2 : (tile == 32 ? 8 : 8);
                check_ss(ss_set_kernel_config(tile, other),
                         "ss_set_kernel_config");
                route();
                check_ss(ss_read_status(d_ws, ws_bytes, stream, nullptr),
                         "cross route");
                ss_set_kernel_config(tile, saved);
                std::vector<uint8_t> cx(n), cn(n);
                check_cuda(cudaMemcpy(cx.data(), d_max, n,
                                      cudaMemcpyDeviceToHost), "D2H");
                check_cuda(cudaMemcpy(cn.data(), d_min, n,
                                      cudaMemcpyDeviceToHost), "D2H");
                cross_max = mismatches(mx, cx);
                cross_min = mismatches(mn, cn);
            }
            uint64_t oracle_max = 0, oracle_min = 0;
            if (!expected_max_dir.empty()) {
                const std::string stem = path.stem().string();
                const auto emax = expected(expected_max_dir, stem, w, h);
                const auto emin = expected(expected_min_dir, stem, w, h);
                if (emax.empty() || emin.empty()) {
                    throw std::runtime_error("no expected masks for " + stem);
                }
                oracle_max = mismatches(mx, emax);
                oracle_min = mismatches(mn, emin);
            }
            total_oracle += oracle_max + oracle_min;
            total_cross += cross_max + cross_min;
            if (save_masks) {
                const std::string stem = path.stem().string();
                check_ss(ss_write_pgm((output_dir / "masks" / (stem + "_max.pgm"))
                                          .string().c_str(),
                                      mx.data(), w, h, w), "ss_write_pgm");
                check_ss(ss_write_pgm((output_dir / "masks" / (stem + "_min.pgm"))
                                          .string().c_str(),
                                      mn.data(), w, h, w), "ss_write_pgm");
            }
            const double px = static_cast<double>(n);
            const double mp = px / 1e6;
            const uint64_t total = 3ull * n + ws_bytes;
            csv << quote("sparse_seam_b200") << ','
                << quote(path.filename().string()) << ',' << w << ',' << h
                << ',' << std::fixed << std::setprecision(6) << mp << ','
                << warmup << ',' << reps << ',' << block << ',' << total
                << ',' << static_cast<double>(total) / px << ',' << ws_bytes
                << ',' << static_cast<double>(ws_bytes) / px << ','
                << t.median_compute_ms << ',' << t.p95_compute_ms << ','
                << mp / (t.median_compute_ms / 1000.0) << ','
                << t.median_h2h_ms << ',' << t.p95_h2h_ms << ','
                << mp / (t.median_h2h_ms / 1000.0) << ',' << 0.0 << ','
                << 0.0 << ',' << oracle_max << ',' << oracle_min << ','
                << cross_max << ',' << cross_min << '\n';
            cudaFreeHost(h_img);
            cudaFreeHost(h_max);
            cudaFreeHost(h_min);
            cudaFree(d_img);
            cudaFree(d_max);
            cudaFree(d_min);
            cudaFree(d_ws);
        }
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        cudaStreamDestroy(stream);
        std::cout << "images=" << files.size()
                  << " oracle_mismatches=" << total_oracle
                  << " cross_mismatches=" << total_cross << "\n";
        return (total_oracle || total_cross) ? 1 : 0;
    } catch (const std::exception& e) {
        std::cerr << "ss_harness: " << e.what() << "\n";
        return 3;
    }
}

// ss_pack.cu -- compact mask transfer for host-to-host use.
//
// Host-to-host throughput is bound by PCIe: 1 byte per pixel goes in and two
// 0/255 mask bytes come back.  The masks carry one bit each, so the device
// packs them into bit planes (a warp loads 32 consecutive mask bytes and
// ballots their non-zero bits into one 32-bit word), the bit planes cross
// the bus (0.25 byte per pixel for both masks), and host threads expand them
// back into 0/255 bytes in the caller's buffers.  The expansion can be
// enqueued on a stream as a host function, so it is ordered after the copy
// that brings the bits and before anything enqueued after it.
//
// No counterpart in the reference, which copies both byte masks back
// (harness/primary/gpu_common_v0_6.cu:351-373).
#include <cuda_runtime.h>
#include <omp.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include "sparse_seam.h"

namespace ss {
namespace pack {

// One warp per group of 8 words (256 mask bytes) per iteration, grid-stride.
__global__ void __launch_bounds__(256)
pack_kernel(const uint8_t* __restrict__ maxima,
            const uint8_t* __restrict__ minima, uint64_t n,
            uint32_t* __restrict__ max_bits, uint32_t* __restrict__ min_bits) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const uint64_t words = (n + 31) / 32;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x +
                           threadIdx.x) >> 5;
    const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t w0 = warp * 8; w0 < words; w0 += warps * 8) {
        uint8_t vx[8];
        uint8_t vn[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint64_t i = (w0 + k) * 32 + lane;
            vx[k] = i < n ? maxima[i] : 0;
            vn[k] = i < n ? minima[i] : 0;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t bx = __ballot_sync(~0u, vx[k] != 0);
            const uint32_t bn = __ballot_sync(~0u, vn[k] != 0);
            if (lane == 0 && w0 + k < words) {
                max_bits[w0 + k] = bx;
                min_bits[w0 + k] = bn;
            }
        }
    }
}

// Bytes 0x00 / 0xFF of the 8 bits of a byte, bit i -> byte i.
struct Table {
    uint64_t v[256];
    Table() {
        for (int b = 0; b < 256; ++b) {
            uint64_t x = 0;
            for (int i = 0; i < 8; ++i) {
                if ((b >> i) & 1) x |= 0xFFull << (8 * i);
            }
            v[b] = x;
        }
    }
};

static const Table& table() {
    static const Table t;
    return t;
}

static inline uint8_t bit_byte(const uint8_t* b8, uint64_t i) {
    return ((b8[i / 8] >> (i % 8)) & 1) ? 255 : 0;
}

// Writes n bytes (bit i of the planes -> byte i).  The output is written
// once and not read back by this thread, so the aligned middle goes out with
// 16-byte streaming stores (no read-for-ownership of the destination lines).
static void expand(const uint32_t* bits, uint64_t n, uint8_t* out,
                   const Table& t) {
    const uint8_t* b8 = reinterpret_cast<const uint8_t*>(bits);
    uint64_t i = 0;
#if defined(__x86_64__)
    const uint64_t mis = reinterpret_cast<uintptr_t>(out) & 15u;
    const uint64_t head = mis ? 16 - mis : 0;
    for (; i < head && i < n; ++i) {
        out[i] = bit_byte(b8, i);
    }
    const unsigned shift = static_cast<unsigned>(i % 8);
    const uint64_t plane_bytes = ((n + 31) / 32) * 4;
    for (; i + 16 <= n; i += 16) {
        // 16 bits starting at bit i lie in bytes at .. at + 2; byte at + 2 is
        // needed only when it holds bit i + 15 (< n), so it exists then.
        const uint64_t at = i / 8;
        const uint32_t w = static_cast<uint32_t>(b8[at]) |
                           (static_cast<uint32_t>(b8[at + 1]) << 8) |
                           (at + 2 < plane_bytes
                                ? static_cast<uint32_t>(b8[at + 2]) << 16
                                : 0u);
        const uint32_t v = w >> shift;
        const __m128i x = _mm_set_epi64x(
            static_cast<long long>(t.v[(v >> 8) & 0xFF]),
            static_cast<long long>(t.v[v & 0xFF]));
        _mm_stream_si128(reinterpret_cast<__m128i*>(out + i), x);
    }
    _mm_sfence();
#endif
    for (; i + 8 <= n && i % 8 == 0; i += 8) {
        std::memcpy(out + i, &t.v[b8[i / 8]], 8);
    }
    for (; i < n; ++i) {
        out[i] = bit_byte(b8, i);
    }
}

#if defined(__x86_64__)
// 64 bits of the planes starting at bit i (i + 64 <= n); bytes beyond the
// planes are read only when they hold a needed bit.
static inline uint64_t bits64(const uint8_t* b8, uint64_t i,
                              uint64_t plane_bytes) {
    const uint64_t at = i / 8;
    const unsigned shift = static_cast<unsigned>(i % 8);
    uint64_t lo;
    std::memcpy(&lo, b8 + at, 8);
    if (shift == 0) {
        return lo;
    }
    const uint64_t hi = at + 8 < plane_bytes ? b8[at + 8] : 0;
    return (lo >> shift) | (hi << (64 - shift));
}

// AVX-512BW: one mask register becomes 64 bytes of 0x00 / 0xFF.
__attribute__((target("avx512f,avx512bw")))
static void expand_avx512(const uint32_t* bits, uint64_t n, uint8_t* out) {
    const uint8_t* b8 = reinterpret_cast<const uint8_t*>(bits);
    const uint64_t plane_bytes = ((n + 31) / 32) * 4;
    uint64_t i = 0;
    const uint64_t mis = reinterpret_cast<uintptr_t>(out) & 63u;
    const uint64_t head = mis ? 64 - mis : 0;
    for (; i < head && i < n; ++i) {
        out[i] = bit_byte(b8, i);
    }
    for (; i + 64 <= n; i += 64) {
        const __m512i x = _mm512_movm_epi8(
            static_cast<__mmask64>(bits64(b8, i, plane_bytes)));
        _mm512_stream_si512(reinterpret_cast<__m512i*>(out + i), x);
    }
    _mm_sfence();
    for (; i < n; ++i) {
        out[i] = bit_byte(b8, i);
    }
}

// AVX2: 32 bits become 32 bytes (each byte picks its bit-byte with a
// shuffle, then tests its own bit).
__attribute__((target("avx2")))
static void expand_avx2(const uint32_t* bits, uint64_t n, uint8_t* out) {
    const uint8_t* b8 = reinterpret_cast<const uint8_t*>(bits);
    const uint64_t plane_bytes = ((n + 31) / 32) * 4;
    const __m256i pick = _mm256_setr_epi8(
        0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1,
        2, 2, 2, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3);
    const __m256i sel = _mm256_set1_epi64x(
        static_cast<long long>(0x8040201008040201ull));
    uint64_t i = 0;
    const uint64_t mis = reinterpret_cast<uintptr_t>(out) & 31u;
    const uint64_t head = mis ? 32 - mis : 0;
    for (; i < head && i < n; ++i) {
        out[i] = bit_byte(b8, i);
    }
    for (; i + 64 <= n; i += 32) {
        const uint32_t w =
            static_cast<uint32_t>(bits64(b8, i, plane_bytes));
        const __m256i v = _mm256_shuffle_epi8(
            _mm256_set1_epi32(static_cast<int>(w)), pick);
        const __m256i x = _mm256_cmpeq_epi8(_mm256_and_si256(v, sel), sel);
        _mm256_stream_si256(reinterpret_cast<__m256i*>(out + i), x);
    }
    _mm_sfence();
    for (; i < n; ++i) {
        out[i] = bit_byte(b8, i);
    }
}

// The widest expansion the CPU supports; SS_UNPACK_SIMD (0 scalar, 1 AVX2,
// 2 AVX-512) caps it, so every path can be tested on one machine.
static int simd_level() {
    static const int level = [] {
        int l = __builtin_cpu_supports("avx512bw") ? 2
                : __builtin_cpu_supports("avx2")   ? 1
                                                   : 0;
        const char* cap = std::getenv("SS_UNPACK_SIMD");
        if (cap && cap[0] >= '0' && cap[0] <= '2' && cap[0] - '0' < l) {
            l = cap[0] - '0';
        }
        return l;
    }();
    return level;
}
#endif

static void expand_best(const uint32_t* bits, uint64_t n, uint8_t* out,
                        const Table& t) {
#if defined(__x86_64__)
    const int level = simd_level();
    if (level == 2) {
        expand_avx512(bits, n, out);
        return;
    }
    if (level == 1) {
        expand_avx2(bits, n, out);
        return;
    }
#endif
    expand(bits, n, out, t);
}

// Threads for an unpack: the caller's choice, else all processors but one
// (the thread that waits for the GPU or feeds it keeps a core; with every
// core busy expanding, the waiting thread and the runtime's own threads
// preempt the expansion threads and the unpack slows several-fold).
static int unpack_threads(int threads) {
    if (threads > 0) {
        return threads;
    }
    const int procs = omp_get_num_procs();
    return procs > 1 ? procs - 1 : 1;
}

// Threads for an enqueued unpack: the caller's choice, else a quarter of the
// processors.  An enqueued expansion runs while the copy engines read the
// next chunks' images from the same host memory; its streaming stores
// (2 bytes per pixel) contend with those reads, and beyond a few threads
// the copies lose more than the expansion gains (on a 16-processor host:
// 7.6 ms per 292 Mpixel pass with 4 threads, 8.1 ms with 15).
static int enqueued_unpack_threads(int threads) {
    if (threads > 0) {
        return threads;
    }
    const int procs = omp_get_num_procs();
    return procs >= 8 ? procs / 4 : (procs > 2 ? 2 : 1);
}

struct UnpackJob {
    const uint32_t* max_bits;
    const uint32_t* min_bits;
    uint64_t n;
    uint8_t* maxima;
    uint8_t* minima;
    int threads;
};

static void unpack(const UnpackJob& j) {
    const Table& t = table();
    // Blocks of 64 Ki pixels (a multiple of 32, so blocks start on words).
    const uint64_t block = 1ull << 16;
    const int64_t blocks = static_cast<int64_t>((j.n + block - 1) / block);
#pragma omp parallel for schedule(static) num_threads(j.threads)
    for (int64_t b = 0; b < 2 * blocks; ++b) {
        const bool is_min = b >= blocks;
        const uint64_t first = static_cast<uint64_t>(is_min ? b - blocks : b) *
                               block;
        const uint64_t count = j.n - first < block ? j.n - first : block;
        expand_best((is_min ? j.min_bits : j.max_bits) + first / 32, count,
                    (is_min ? j.minima : j.maxima) + first, t);
    }
}

static void CUDART_CB unpack_callback(void* data) {
    UnpackJob* j = static_cast<UnpackJob*>(data);
    unpack(*j);
    delete j;
}

}  // namespace pack
}  // namespace ss

using namespace ss::pack;

extern "C" {

ss_status ss_pack_masks(const uint8_t* d_maxima, const uint8_t* d_minima,
                        uint64_t n, uint32_t* d_max_bits, uint32_t* d_min_bits,
                        void* stream) {
    if (!d_maxima || !d_minima || !d_max_bits || !d_min_bits) {
        return SS_ERR_INVALID_VALUE;
    }
    if (reinterpret_cast<uintptr_t>(d_max_bits) % 4 ||
        reinterpret_cast<uintptr_t>(d_min_bits) % 4) {
        return SS_ERR_MISALIGNED;
    }
    if (n == 0) {
        return SS_OK;
    }
    (void)cudaGetLastError();
    const uint64_t groups = ((n + 31) / 32 + 7) / 8;   // warps of work
    const uint64_t want = (groups + 7) / 8;             // 8 warps per CTA
    int device = 0;
    int sms = 148;
    if (cudaGetDevice(&device) == cudaSuccess) {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    }
    const uint64_t cap = static_cast<uint64_t>(sms) * 8;
    const unsigned grid = static_cast<unsigned>(want < cap ? want : cap);
    pack_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        d_maxima, d_minima, n, d_max_bits, d_min_bits);
    return cudaGetLastError() == cudaSuccess ? SS_OK : SS_ERR_CUDA;
}

ss_status ss_unpack_masks(const uint32_t* h_max_bits,
                          const uint32_t* h_min_bits, uint64_t n,
                          uint8_t* h_maxima, uint8_t* h_minima, int threads) {
    if (!h_max_bits || !h_min_bits || !h_maxima || !h_minima) {
        return SS_ERR_INVALID_VALUE;
    }
    UnpackJob j{h_max_bits, h_min_bits, n, h_maxima, h_minima,
                unpack_threads(threads)};
    unpack(j);
    return SS_OK;
}

ss_status ss_enqueue_unpack_masks(const uint32_t* h_max_bits,
                                  const uint32_t* h_min_bits, uint64_t n,
                                  uint8_t* h_maxima, uint8_t* h_minima,
                                  int threads, void* stream) {
    if (!h_max_bits || !h_min_bits || !h_maxima || !h_minima) {
        return SS_ERR_INVALID_VALUE;
    }
    UnpackJob* j = new (std::nothrow)
        UnpackJob{h_max_bits, h_min_bits, n, h_maxima, h_minima,
                  enqueued_unpack_threads(threads)};
    if (!j) {
        return SS_ERR_HOST_ALLOC;
    }
    if (cudaLaunchHostFunc(static_cast<cudaStream_t>(stream), unpack_callback,
                           j) != cudaSuccess) {
        delete j;
        return SS_ERR_CUDA;
    }
    return SS_OK;
}

}  // extern "C"

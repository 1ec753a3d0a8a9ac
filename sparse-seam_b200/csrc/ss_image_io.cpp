// ss_image_io.cpp -- 8-bit grayscale image files for the harness and the
// serving loop: PGM (P5 binary, P2 ASCII) and PNG (every colour type, bit
// depths 1, 2, 4 and 8, all five scanline filters, not interlaced), read as
// one byte per pixel; PGM (P5) written.
//
// The reference reads images with OpenCV, cv::imread(path,
// IMREAD_GRAYSCALE) (harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:87-103,
// :941-942).  For PNG that decoder asks libpng for gray output: samples of
// 1, 2 or 4 bits are scaled to 0..255, alpha is dropped, a palette is
// expanded, and colour is converted with the weights (0.299, 0.587) held as
// 15-bit fractions, truncated: red (29900 << 15) / 100000 = 9797, green
// (58700 << 15) / 100000 = 19234, blue the rest of 32768 = 3737, and
// gray = (9797 R + 19234 G + 3737 B) >> 15 without rounding (checked equal to
// OpenCV 4.13's result on 65,536 random colours).  The same steps are
// restated here with zlib for the decompression.
#include <zlib.h>

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sparse_seam.h"

namespace {

bool read_file(const char* path, std::vector<uint8_t>& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 0) {
        std::fclose(f);
        return false;
    }
    out.resize(static_cast<size_t>(size));
    const size_t got = size ? std::fread(out.data(), 1, out.size(), f) : 0;
    std::fclose(f);
    return got == out.size();
}

// ---- PGM -------------------------------------------------------------------

// Next header token, skipping whitespace and '#' comments.
bool pgm_token(const std::vector<uint8_t>& d, size_t& pos, long& value) {
    for (;;) {
        while (pos < d.size() && std::isspace(d[pos])) ++pos;
        if (pos < d.size() && d[pos] == '#') {
            while (pos < d.size() && d[pos] != '\n') ++pos;
            continue;
        }
        break;
    }
    if (pos >= d.size() || !std::isdigit(d[pos])) return false;
    value = 0;
    while (pos < d.size() && std::isdigit(d[pos])) {
        value = value * 10 + (d[pos] - '0');
        if (value > (1L << 30)) return false;
        ++pos;
    }
    return true;
}

ss_status decode_pgm(const std::vector<uint8_t>& d, std::vector<uint8_t>& px,
                     int& w, int& h) {
    if (d.size() < 2 || d[0] != 'P' || (d[1] != '5' && d[1] != '2')) {
        return SS_ERR_INVALID_VALUE;
    }
    size_t pos = 2;
    long width, height, maxval;
    if (!pgm_token(d, pos, width) || !pgm_token(d, pos, height) ||
        !pgm_token(d, pos, maxval) || width < 1 || height < 1 ||
        maxval < 1 || maxval > 255) {
        return SS_ERR_INVALID_VALUE;
    }
    const size_t n = static_cast<size_t>(width) * static_cast<size_t>(height);
    px.resize(n);
    if (d[1] == '5') {
        ++pos;   // the single whitespace byte after maxval
        if (d.size() < pos + n) return SS_ERR_INVALID_VALUE;
        std::memcpy(px.data(), d.data() + pos, n);
    } else {
        for (size_t i = 0; i < n; ++i) {
            long v;
            if (!pgm_token(d, pos, v) || v > maxval) {
                return SS_ERR_INVALID_VALUE;
            }
            px[i] = static_cast<uint8_t>(v);
        }
    }
    if (maxval != 255) {
        // OpenCV scales a smaller maxval to 0..255 (value * 255 / maxval,
        // rounded).
        for (auto& v : px) {
            v = static_cast<uint8_t>((v * 255 + maxval / 2) / maxval);
        }
    }
    w = static_cast<int>(width);
    h = static_cast<int>(height);
    return SS_OK;
}

// ---- PNG -------------------------------------------------------------------

uint32_t be32(const uint8_t* p) {
    return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) |
           (uint32_t(p[2]) << 8) | uint32_t(p[3]);
}

int paeth(int a, int b, int c) {
    const int p = a + b - c;
    const int pa = p > a ? p - a : a - p;
    const int pb = p > b ? p - b : b - p;
    const int pc = p > c ? p - c : c - p;
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

uint8_t rgb_gray(int r, int g, int b) {
    return static_cast<uint8_t>((9797 * r + 19234 * g + 3737 * b) >> 15);
}

ss_status decode_png(const std::vector<uint8_t>& d, std::vector<uint8_t>& px,
                     int& w, int& h) {
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (d.size() < 8 || std::memcmp(d.data(), sig, 8) != 0) {
        return SS_ERR_INVALID_VALUE;
    }
    size_t pos = 8;
    uint32_t width = 0, height = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat;
    std::vector<uint8_t> palette;
    bool ihdr = false;
    while (pos + 12 <= d.size()) {
        const uint32_t len = be32(d.data() + pos);
        const uint8_t* type = d.data() + pos + 4;
        const uint8_t* body = d.data() + pos + 8;
        if (len > d.size() - pos - 12) return SS_ERR_INVALID_VALUE;
        if (!std::memcmp(type, "IHDR", 4) && len >= 13) {
            width = be32(body);
            height = be32(body + 4);
            depth = body[8];
            ctype = body[9];
            interlace = body[12];
            ihdr = true;
        } else if (!std::memcmp(type, "PLTE", 4)) {
            palette.assign(body, body + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), body, body + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        pos += 12 + len;
    }
    if (!ihdr || width < 1 || height < 1 || width > (1u << 30) ||
        height > (1u << 30) || interlace != 0) {
        return SS_ERR_INVALID_VALUE;
    }
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: return SS_ERR_INVALID_VALUE;
    }
    const bool small = depth == 1 || depth == 2 || depth == 4;
    if (!(depth == 8 || (small && (ctype == 0 || ctype == 3)))) {
        return SS_ERR_INVALID_VALUE;   // 16-bit samples are not 8-bit images
    }
    if (ctype == 3 && (palette.empty() || palette.size() % 3)) {
        return SS_ERR_INVALID_VALUE;
    }
    const size_t row_bytes =
        (static_cast<size_t>(width) * channels * depth + 7) / 8;
    const size_t stride = row_bytes + 1;
    if (stride * height > 0xFFFFFFFFull || idat.size() > 0xFFFFFFFFull) {
        return SS_ERR_TOO_LARGE;   // beyond one zlib call's 32-bit counters
    }
    std::vector<uint8_t> raw(stride * height);
    z_stream zs{};
    if (inflateInit(&zs) != Z_OK) return SS_ERR_HOST_ALLOC;
    zs.next_in = idat.data();
    zs.avail_in = static_cast<uInt>(idat.size());
    zs.next_out = raw.data();
    zs.avail_out = static_cast<uInt>(raw.size());
    const int zr = inflate(&zs, Z_FINISH);
    const size_t produced = raw.size() - zs.avail_out;
    inflateEnd(&zs);
    if ((zr != Z_STREAM_END && zr != Z_OK && zr != Z_BUF_ERROR) ||
        produced != raw.size()) {
        return SS_ERR_INVALID_VALUE;
    }
    // Undo the scanline filters in place (bpp = bytes per complete pixel,
    // at least 1).
    const size_t bpp = depth == 8 ? static_cast<size_t>(channels) : 1;
    std::vector<uint8_t> prev(row_bytes, 0);
    for (uint32_t y = 0; y < height; ++y) {
        uint8_t* row = raw.data() + y * stride;
        const int filter = row[0];
        uint8_t* cur = row + 1;
        for (size_t i = 0; i < row_bytes; ++i) {
            const int a = i >= bpp ? cur[i - bpp] : 0;
            const int b = prev[i];
            const int c = i >= bpp ? prev[i - bpp] : 0;
            int v = cur[i];
            switch (filter) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) >> 1; break;
                case 4: v += paeth(a, b, c); break;
                default: return SS_ERR_INVALID_VALUE;
            }
            cur[i] = static_cast<uint8_t>(v);
        }
        std::memcpy(prev.data(), cur, row_bytes);
    }
    px.resize(static_cast<size_t>(width) * height);
    const size_t colors = palette.size() / 3;
    for (uint32_t y = 0; y < height; ++y) {
        const uint8_t* s = raw.data() + y * stride + 1;
        uint8_t* o = px.data() + static_cast<size_t>(y) * width;
        for (uint32_t x = 0; x < width; ++x) {
            int sample;   // gray value or palette index
            if (small) {
                const int per = 8 / depth;
                const int shift = (per - 1 - static_cast<int>(x % per)) * depth;
                sample = (s[x / per] >> shift) & ((1 << depth) - 1);
                if (ctype == 0) {
                    sample = sample * 255 / ((1 << depth) - 1);
                }
            } else {
                sample = s[static_cast<size_t>(x) * channels];
            }
            switch (ctype) {
                case 0:
                case 4:
                    o[x] = static_cast<uint8_t>(sample);
                    break;
                case 2:
                case 6: {
                    const uint8_t* p = s + static_cast<size_t>(x) * channels;
                    o[x] = rgb_gray(p[0], p[1], p[2]);
                    break;
                }
                case 3: {
                    if (static_cast<size_t>(sample) >= colors) {
                        return SS_ERR_INVALID_VALUE;
                    }
                    const uint8_t* p = palette.data() + 3 * sample;
                    o[x] = rgb_gray(p[0], p[1], p[2]);
                    break;
                }
            }
        }
    }
    w = static_cast<int>(width);
    h = static_cast<int>(height);
    return SS_OK;
}

}  // namespace

extern "C" {

ss_status ss_read_image(const char* path, uint8_t* pixels, size_t capacity,
                        int* width, int* height) {
    if (!path || !width || !height) {
        return SS_ERR_INVALID_VALUE;
    }
    std::vector<uint8_t> data;
    if (!read_file(path, data)) {
        return SS_ERR_INVALID_VALUE;
    }
    std::vector<uint8_t> px;
    int w = 0, h = 0;
    ss_status st;
    if (data.size() >= 8 && data[0] == 137 && data[1] == 'P') {
        st = decode_png(data, px, w, h);
    } else {
        st = decode_pgm(data, px, w, h);
    }
    if (st != SS_OK) {
        return st;
    }
    *width = w;
    *height = h;
    if (!pixels) {
        return SS_OK;   // size query
    }
    if (capacity < px.size()) {
        return SS_ERR_WORKSPACE_TOO_SMALL;
    }
    std::memcpy(pixels, px.data(), px.size());
    return SS_OK;
}

ss_status ss_write_pgm(const char* path, const uint8_t* pixels, int width,
                       int height, int pitch) {
    if (!path || !pixels || width < 1 || height < 1 || pitch < width) {
        return SS_ERR_INVALID_VALUE;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        return SS_ERR_INVALID_VALUE;
    }
    std::fprintf(f, "P5\n%d %d\n255\n", width, height);
    bool ok = true;
    for (int y = 0; y < height && ok; ++y) {
        ok = std::fwrite(pixels + static_cast<size_t>(y) * pitch, 1,
                         static_cast<size_t>(width), f) ==
             static_cast<size_t>(width);
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? SS_OK : SS_ERR_INVALID_VALUE;
}

}  // extern "C"

// ss_image_io.cpp -- 8-bit grayscale image files for the harness and the
// serving loop: PGM (P5 binary, P2 ASCII), PNG (every colour type, bit
// depths 1, 2, 4 and 8, all five scanline filters, not interlaced) and BMP
// (1-, 4- and 8-bit palettes, 16-bit 5-5-5 / 5-6-5, 24- and 32-bit, RLE8 and
// RLE4, core and V1-V5 headers), read as one byte per pixel; PGM (P5)
// written.
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

// ---- BMP -------------------------------------------------------------------
// OpenCV's BMP decoder converts colour itself, with the weights
// (0.114, 0.587, 0.299) for (B, G, R) held as 14-bit fractions and rounded:
// gray = (1868 B + 9617 G + 4899 R + 8192) >> 14 (checked equal to OpenCV
// 4.13 on 65,536 random colours).  A palette is converted entry by entry;
// 5- and 6-bit fields are widened by a shift (no low-bit copy); pixels that
// an RLE stream skips take palette entry 0.  32-bit pixels with bit fields
// in a V3 or later header take a float path instead:
// gray = (int)((0.299f R + 0.587f G) + 0.114f B) in single precision, each
// step rounded, truncated at the end (equal to OpenCV 4.13 on all 2^24
// colours).

uint32_t le16(const uint8_t* p) {
    return uint32_t(p[0]) | (uint32_t(p[1]) << 8);
}

uint32_t le32(const uint8_t* p) {
    return le16(p) | (le16(p + 2) << 16);
}

uint8_t bgr_gray(int b, int g, int r) {
    return static_cast<uint8_t>((1868 * b + 9617 * g + 4899 * r + 8192) >> 14);
}

uint8_t bgr_gray_float(int b, int g, int r) {
    // Separate statements and volatile keep each product and sum rounded to
    // single precision (no fused multiply-add).
    volatile float t = 0.299f * static_cast<float>(r);
    volatile float u = 0.587f * static_cast<float>(g);
    t = t + u;
    u = 0.114f * static_cast<float>(b);
    t = t + u;
    const int v = static_cast<int>(t);
    return static_cast<uint8_t>(v > 255 ? 255 : v);
}

ss_status decode_bmp(const std::vector<uint8_t>& d, std::vector<uint8_t>& px,
                     int& w, int& h) {
    const size_t n = d.size();
    if (n < 26 || d[0] != 'B' || d[1] != 'M') {
        return SS_ERR_INVALID_VALUE;
    }
    const size_t off = le32(&d[10]);
    const size_t hs = le32(&d[14]);
    int64_t width = 0, height = 0;
    uint32_t bpp = 0, comp = 0, ncolors = 0;
    uint32_t masks[3] = {0, 0, 0};
    size_t pal_at = 14 + hs;
    size_t pal_entry = 4;
    if (hs == 12) {   // OS/2 core header: 16-bit sizes, 3-byte palette
        width = le16(&d[18]);
        height = static_cast<int16_t>(le16(&d[20]));
        bpp = le16(&d[24]);
        pal_entry = 3;
    } else if (hs >= 40 && hs <= 124 && n >= 14 + hs) {
        width = static_cast<int32_t>(le32(&d[18]));
        height = static_cast<int32_t>(le32(&d[22]));
        bpp = le16(&d[28]);
        comp = le32(&d[30]);
        ncolors = le32(&d[46]);
        if (comp == 3) {
            // Bit fields: inside a V2+ header, else the 12 bytes after it.
            size_t at = 54;
            if (hs == 40) {
                pal_at += 12;
            }
            if (n < at + 12) {
                return SS_ERR_INVALID_VALUE;
            }
            for (int k = 0; k < 3; ++k) {
                masks[k] = le32(&d[at + 4 * k]);
            }
        }
    } else {
        return SS_ERR_INVALID_VALUE;
    }
    const bool top_down = height < 0;
    if (top_down) {
        height = -height;
    }
    if (width <= 0 || height <= 0 || width * height > (int64_t(1) << 31)) {
        return SS_ERR_INVALID_VALUE;
    }
    // Gray value of each palette index (indices past the palette give 0).
    uint8_t gray_pal[256] = {0};
    if (bpp <= 8) {
        const uint32_t cap = 1u << bpp;
        const uint32_t count = ncolors && ncolors < cap ? ncolors : cap;
        if (pal_at + size_t(count) * pal_entry > n) {
            return SS_ERR_INVALID_VALUE;
        }
        for (uint32_t i = 0; i < count; ++i) {
            const uint8_t* e = &d[pal_at + size_t(i) * pal_entry];
            gray_pal[i] = bgr_gray(e[0], e[1], e[2]);
        }
    }
    const size_t W = static_cast<size_t>(width);
    const size_t H = static_cast<size_t>(height);
    px.assign(W * H, gray_pal[0]);
    auto row_of = [&](size_t file_row) -> uint8_t* {
        return px.data() + (top_down ? file_row : H - 1 - file_row) * W;
    };
    if (comp == 1 || comp == 2) {
        // RLE8 / RLE4: (count, index) runs; escapes 0 = end of line, 1 = end
        // of bitmap, 2 = move by (dx, dy), n >= 3 = n literal indices padded
        // to a 16-bit boundary.
        const bool rle4 = comp == 2;
        if (bpp != (rle4 ? 4u : 8u) || top_down) {
            return SS_ERR_INVALID_VALUE;
        }
        size_t pos = off, x = 0, y = 0;
        while (y < H) {
            if (pos + 2 > n) {
                return SS_ERR_INVALID_VALUE;
            }
            const uint32_t cnt = d[pos], c = d[pos + 1];
            pos += 2;
            if (cnt > 0) {
                if (x + cnt > W) {
                    return SS_ERR_INVALID_VALUE;
                }
                uint8_t* o = row_of(y);
                for (uint32_t i = 0; i < cnt; ++i, ++x) {
                    const uint32_t idx =
                        rle4 ? ((i & 1u) ? (c & 15u) : (c >> 4)) : c;
                    o[x] = gray_pal[idx];
                }
            } else if (c == 0) {
                x = 0;
                ++y;
            } else if (c == 1) {
                break;
            } else if (c == 2) {
                if (pos + 2 > n) {
                    return SS_ERR_INVALID_VALUE;
                }
                x += d[pos];
                y += d[pos + 1];
                pos += 2;
                if (x > W) {
                    return SS_ERR_INVALID_VALUE;
                }
            } else {
                const size_t bytes = rle4 ? (c + 1) / 2 : c;
                if (x + c > W || pos + bytes > n) {
                    return SS_ERR_INVALID_VALUE;
                }
                uint8_t* o = row_of(y);
                for (uint32_t i = 0; i < c; ++i, ++x) {
                    const uint8_t b = d[pos + (rle4 ? i / 2 : i)];
                    const uint32_t idx =
                        rle4 ? ((i & 1u) ? (b & 15u) : (b >> 4)) : b;
                    o[x] = gray_pal[idx];
                }
                pos += (bytes + 1) & ~size_t(1);
            }
        }
        w = static_cast<int>(width);
        h = static_cast<int>(height);
        return SS_OK;
    }
    // Uncompressed rows, each padded to 4 bytes.
    // 0 palette, 1 = 555, 2 = 565, 3 = BGR, 4 = BGRx, 5 = BGRx (float)
    int format = -1;
    if (comp == 0) {
        format = bpp <= 8 && (bpp == 1 || bpp == 4 || bpp == 8) ? 0
               : bpp == 16 ? 1 : bpp == 24 ? 3 : bpp == 32 ? 4 : -1;
    } else if (comp == 3) {
        if (bpp == 16 && masks[0] == 0x7C00u && masks[1] == 0x03E0u &&
            masks[2] == 0x001Fu) {
            format = 1;
        } else if (bpp == 16 && masks[0] == 0xF800u && masks[1] == 0x07E0u &&
                   masks[2] == 0x001Fu) {
            format = 2;
        } else if (bpp == 32 && masks[0] == 0x00FF0000u &&
                   masks[1] == 0x0000FF00u && masks[2] == 0x000000FFu) {
            format = hs >= 56 ? 5 : 4;
        }
    }
    if (format < 0) {
        return SS_ERR_INVALID_VALUE;
    }
    const size_t stride = (W * bpp + 31) / 32 * 4;
    if (off > n || (n - off) / stride < H) {
        return SS_ERR_INVALID_VALUE;
    }
    for (size_t r = 0; r < H; ++r) {
        const uint8_t* s = &d[off + r * stride];
        uint8_t* o = row_of(r);
        for (size_t x = 0; x < W; ++x) {
            switch (format) {
                case 0: {
                    const size_t bit = x * bpp;
                    const uint32_t idx =
                        (s[bit / 8] >> (8 - bpp - bit % 8)) & ((1u << bpp) - 1u);
                    o[x] = gray_pal[idx];
                    break;
                }
                case 1: {
                    const uint32_t t = le16(s + 2 * x);
                    o[x] = bgr_gray((t << 3) & 0xF8, (t >> 2) & 0xF8,
                                    (t >> 7) & 0xF8);
                    break;
                }
                case 2: {
                    const uint32_t t = le16(s + 2 * x);
                    o[x] = bgr_gray((t << 3) & 0xF8, (t >> 3) & 0xFC,
                                    (t >> 8) & 0xF8);
                    break;
                }
                case 3:
                    o[x] = bgr_gray(s[3 * x], s[3 * x + 1], s[3 * x + 2]);
                    break;
                case 4:
                    o[x] = bgr_gray(s[4 * x], s[4 * x + 1], s[4 * x + 2]);
                    break;
                default:
                    o[x] = bgr_gray_float(s[4 * x], s[4 * x + 1], s[4 * x + 2]);
                    break;
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
    } else if (data.size() >= 2 && data[0] == 'B' && data[1] == 'M') {
        st = decode_bmp(data, px, w, h);
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

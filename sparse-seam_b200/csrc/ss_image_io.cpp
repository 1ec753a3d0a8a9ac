// ss_image_io.cpp -- 8-bit grayscale image files for the harness and the
// serving loop: PGM (P5 binary, P2 ASCII), PNG (every colour type, bit
// depths 1, 2, 4 and 8, all five scanline filters, not interlaced), BMP
// (1-, 4- and 8-bit palettes, 16-bit 5-5-5 / 5-6-5, 24- and 32-bit, RLE8 and
// RLE4, core and V1-V5 headers), JPEG (baseline / extended sequential /
// progressive Huffman, 8-bit, gray or YCbCr, any sampling, restart
// intervals, EXIF orientation) and TIFF (strips or tiles; none, LZW, Deflate, PackBits;
// predictor; 1/8/16-bit gray, 8-bit RGB(A) and palette; orientation), read as
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

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
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

// ---- JPEG ------------------------------------------------------------------
// Baseline, extended sequential and progressive Huffman JPEG, 8-bit
// samples.  OpenCV asks
// its JPEG library for gray output, which for a YCbCr (or one-component)
// file is the luma plane itself: the Y blocks are entropy-decoded,
// dequantised and inverse-transformed, the chroma blocks only decoded to
// keep the bit stream in step.  The inverse DCT is the Loeffler-Ligtenberg-
// Moschytz factorisation in the fixed point of the IJG "islow" method:
// constants x 2^13, two extra fraction bits between the column and the row
// pass, rounding shifts, and the output offset by 128 and limited through a
// 10-bit wrap-around table.  The EXIF orientation tag is applied as imread
// applies it.  Lossless, arithmetic-coded and 12-bit files, and colour
// spaces other than YCbCr / gray, are refused.

struct JpegHuff {
    int maxcode[18];
    int valptr[17];
    int mincode[17];
    uint8_t vals[256];
    bool defined = false;
};

bool build_huff(const uint8_t* counts, const uint8_t* vals, int nvals,
                JpegHuff& h) {
    int code = 0, k = 0;
    for (int len = 1; len <= 16; ++len) {
        h.valptr[len] = k;
        h.mincode[len] = code;
        code += counts[len - 1];
        k += counts[len - 1];
        h.maxcode[len] = counts[len - 1] ? code - 1 : -1;
        if (code > (1 << len)) {
            return false;
        }
        code <<= 1;
    }
    h.maxcode[17] = 0x7FFFFFFF;
    if (k != nvals || k > 256) {
        return false;
    }
    std::memcpy(h.vals, vals, static_cast<size_t>(k));
    h.defined = true;
    return true;
}

// Entropy-coded data: 0xFF 0x00 is a data byte 0xFF; any other 0xFF xx is a
// marker, after which the reader returns zero bits and `short_data` records
// that a bit past the segment was used (the file is then refused).
struct JpegBits {
    const uint8_t* d;
    size_t n;
    size_t pos;
    uint32_t acc = 0;
    int cnt = 0;
    int real = 0;   // bits of `acc` that came from the segment
    bool at_marker = false;
    bool short_data = false;

    void take(int k) {
        if (k > real) {
            short_data = true;
            real = 0;
        } else {
            real -= k;
        }
    }

    void fill() {
        while (cnt <= 24) {
            uint32_t b = 0;
            if (pos >= n) {
                at_marker = true;   // the file ends inside the segment
            }
            if (!at_marker) {
                b = d[pos];
                if (b == 0xFF) {
                    const uint32_t next = pos + 1 < n ? d[pos + 1] : 0xD9;
                    if (next == 0x00) {
                        pos += 2;
                    } else {
                        at_marker = true;
                        b = 0;
                    }
                } else {
                    ++pos;
                }
            }
            acc |= b << (24 - cnt);
            if (!at_marker) {
                real += 8;
            }
            cnt += 8;
        }
    }
    int bits(int k) {
        if (k == 0) {
            return 0;
        }
        fill();
        const int v = static_cast<int>(acc >> (32 - k));
        acc <<= k;
        cnt -= k;
        take(k);
        return v;
    }
    int decode(const JpegHuff& h) {
        fill();
        int code = 0;
        for (int len = 1; len <= 16; ++len) {
            code = (code << 1) | static_cast<int>(acc >> 31);
            acc <<= 1;
            --cnt;
            take(1);
            if (code <= h.maxcode[len]) {
                return h.vals[h.valptr[len] + code - h.mincode[len]];
            }
        }
        return -1;
    }
    // Skips to the byte after the next RSTn marker (restart interval end).
    bool restart() {
        acc = 0;
        cnt = 0;
        real = 0;
        at_marker = false;
        while (pos + 1 < n) {
            if (d[pos] == 0xFF && d[pos + 1] >= 0xD0 && d[pos + 1] <= 0xD7) {
                pos += 2;
                return true;
            }
            if (d[pos] == 0xFF && d[pos + 1] != 0x00 && d[pos + 1] != 0xFF) {
                return false;
            }
            ++pos;
        }
        return false;
    }
};

int extend(int v, int t) {
    return v < (1 << (t - 1)) ? v - (1 << t) + 1 : v;
}

const uint8_t kZigzag[64] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// Output sample of a row-pass value: + 128, limited to 0..255 through a
// 10-bit wrap (values beyond +-512 wrap as the IJG table does).
uint8_t idct_limit(int64_t x) {
    const int v = static_cast<int>(x & 1023);
    if (v < 128) return static_cast<uint8_t>(v + 128);
    if (v < 512) return 255;
    if (v < 896) return 0;
    return static_cast<uint8_t>(v - 896);
}

// 8 x 8 inverse DCT of dequantised coefficients (natural order) into
// `out` (row stride `stride`).
void idct_islow(const int64_t* in, uint8_t* out, size_t stride) {
    // sqrt(2) times cosine combinations (c_k = cos(k pi / 16)), x 2^13:
    constexpr int64_t k0_298 = 2446;    // -c1 + c3 + c5 - c7
    constexpr int64_t k0_390 = 3196;    // c3 - c5
    constexpr int64_t k0_541 = 4433;    // c6
    constexpr int64_t k0_765 = 6270;    // c2 - c6
    constexpr int64_t k0_899 = 7373;    // c3 - c7
    constexpr int64_t k1_175 = 9633;    // c3
    constexpr int64_t k1_501 = 12299;   // c1 + c3 - c5 - c7
    constexpr int64_t k1_847 = 15137;   // c2 + c6
    constexpr int64_t k1_961 = 16069;   // c3 + c5
    constexpr int64_t k2_053 = 16819;   // c1 + c3 - c5 + c7
    constexpr int64_t k2_562 = 20995;   // c1 + c3
    constexpr int64_t k3_072 = 25172;   // c1 + c3 + c5 - c7
    constexpr int kConst = 13, kPass1 = 2;
    auto descale = [](int64_t x, int nb) -> int64_t {
        return (x + (int64_t(1) << (nb - 1))) >> nb;
    };
    // One 8-point transform: x[0..7] in, y[0..7] before the final shift.
    auto butterfly = [&](const int64_t* x, int64_t* y) {
        int64_t z2 = x[2], z3 = x[6];
        int64_t z1 = (z2 + z3) * k0_541;
        const int64_t t2 = z1 - z3 * k1_847;
        const int64_t t3 = z1 + z2 * k0_765;
        // Multiplications, not shifts: the sums may be negative.
        const int64_t t0 = (x[0] + x[4]) * (int64_t(1) << kConst);
        const int64_t t1 = (x[0] - x[4]) * (int64_t(1) << kConst);
        const int64_t t10 = t0 + t3, t13 = t0 - t3;
        const int64_t t11 = t1 + t2, t12 = t1 - t2;
        int64_t o0 = x[7], o1 = x[5], o2 = x[3], o3 = x[1];
        z1 = o0 + o3;
        z2 = o1 + o2;
        z3 = o0 + o2;
        int64_t z4 = o1 + o3;
        const int64_t z5 = (z3 + z4) * k1_175;
        o0 *= k0_298;
        o1 *= k2_053;
        o2 *= k3_072;
        o3 *= k1_501;
        z1 *= -k0_899;
        z2 *= -k2_562;
        z3 = z3 * -k1_961 + z5;
        z4 = z4 * -k0_390 + z5;
        o0 += z1 + z3;
        o1 += z2 + z4;
        o2 += z2 + z3;
        o3 += z1 + z4;
        y[0] = t10 + o3;
        y[7] = t10 - o3;
        y[1] = t11 + o2;
        y[6] = t11 - o2;
        y[2] = t12 + o1;
        y[5] = t12 - o1;
        y[3] = t13 + o0;
        y[4] = t13 - o0;
    };
    int64_t ws[64];
    for (int c = 0; c < 8; ++c) {   // columns
        int64_t x[8], y[8];
        for (int r = 0; r < 8; ++r) {
            x[r] = in[r * 8 + c];
        }
        butterfly(x, y);
        for (int r = 0; r < 8; ++r) {
            ws[r * 8 + c] = descale(y[r], kConst - kPass1);
        }
    }
    for (int r = 0; r < 8; ++r) {   // rows
        int64_t y[8];
        butterfly(ws + r * 8, y);
        for (int c = 0; c < 8; ++c) {
            out[r * stride + c] =
                idct_limit(descale(y[c], kConst + kPass1 + 3));
        }
    }
}

// One block of a scan into c (natural order, coefficients before
// dequantisation).  Sequential files: the whole block.  Progressive files
// (ITU-T T.81 G.1.2): a DC first scan sets the DC term to the running
// prediction << Al, a DC refinement ORs in bit Al; an AC first scan sets band
// Ss..Se (value << Al) with end-of-band runs spanning blocks; an AC
// refinement adds bit Al to the band's nonzero terms (one correction bit
// each, in zig-zag order) and places new +-2^Al terms after the given
// number of zero terms.
bool decode_block(JpegBits& br, int32_t* c, bool progressive, int ss, int se,
                  int ah, int al, const JpegHuff& dct, const JpegHuff& act,
                  int64_t& pred, int64_t& eobrun) {
    if (!progressive || ss == 0) {
        if (progressive && ah > 0) {
            if (br.bits(1)) {
                c[0] |= 1 << al;
            }
        } else {
            const int t = dct.defined ? br.decode(dct) : -1;
            if (t < 0 || t > 11) {
                return false;
            }
            pred += t ? extend(br.bits(t), t) : 0;
            c[0] = static_cast<int32_t>(pred * (int64_t(1) << al));
        }
        if (progressive) {
            return true;
        }
        for (int z = 1; z < 64;) {
            const int rs = br.decode(act);
            if (rs < 0) {
                return false;
            }
            const int r = rs >> 4, sz = rs & 15;
            if (sz == 0) {
                if (r != 15) break;   // end of block
                z += 16;
                continue;
            }
            z += r;
            if (z > 63) {
                return false;
            }
            c[kZigzag[z]] = extend(br.bits(sz), sz);
            ++z;
        }
        return true;
    }
    if (ah == 0) {   // AC first scan
        if (eobrun > 0) {
            --eobrun;
            return true;
        }
        for (int k = ss; k <= se; ++k) {
            const int rs = br.decode(act);
            if (rs < 0) {
                return false;
            }
            const int r = rs >> 4, sz = rs & 15;
            if (sz) {
                k += r;
                if (k > se) {
                    return false;
                }
                c[kZigzag[k]] =
                    static_cast<int32_t>(extend(br.bits(sz), sz) * (1 << al));
            } else if (r < 15) {
                eobrun = (int64_t(1) << r) - 1 + (r ? br.bits(r) : 0);
                break;
            } else {
                k += 15;
            }
        }
        return true;
    }
    // AC refinement.
    const int32_t p1 = 1 << al, m1 = -p1;
    auto refine = [&](int32_t& v) {
        if (br.bits(1) && (v & p1) == 0) {
            v += v >= 0 ? p1 : m1;
        }
    };
    int k = ss;
    if (eobrun == 0) {
        for (; k <= se; ++k) {
            const int rs = br.decode(act);
            if (rs < 0) {
                return false;
            }
            int r = rs >> 4;
            const int sz = rs & 15;
            int32_t value = 0;
            if (sz) {
                if (sz != 1) {
                    return false;
                }
                value = br.bits(1) ? p1 : m1;
            } else if (r != 15) {
                eobrun = (int64_t(1) << r) + (r ? br.bits(r) : 0);
                break;
            }
            // Skip r zero terms (refining the nonzero ones met on the way),
            // then place the new term, if any.
            for (; k <= se; ++k) {
                int32_t& v = c[kZigzag[k]];
                if (v != 0) {
                    refine(v);
                } else if (r-- == 0) {
                    break;
                }
            }
            if (value) {
                if (k > se) {
                    return false;
                }
                c[kZigzag[k]] = value;
            }
        }
    }
    if (eobrun > 0) {
        for (; k <= se; ++k) {
            int32_t& v = c[kZigzag[k]];
            if (v != 0) {
                refine(v);
            }
        }
        --eobrun;
    }
    return true;
}

// EXIF orientation (tag 0x0112 of IFD0) from an APP1 payload, 1 if none.
int exif_orientation(const uint8_t* p, size_t len) {
    if (len < 14 || std::memcmp(p, "Exif\0\0", 6) != 0) {
        return 1;
    }
    const uint8_t* t = p + 6;
    const size_t tn = len - 6;
    const bool le = t[0] == 'I' && t[1] == 'I';
    if (!le && !(t[0] == 'M' && t[1] == 'M')) {
        return 1;
    }
    auto u16 = [&](size_t at) -> uint32_t {
        return le ? uint32_t(t[at]) | (uint32_t(t[at + 1]) << 8)
                  : (uint32_t(t[at]) << 8) | uint32_t(t[at + 1]);
    };
    auto u32 = [&](size_t at) -> uint32_t {
        return le ? u16(at) | (u16(at + 2) << 16)
                  : (u16(at) << 16) | u16(at + 2);
    };
    const size_t ifd = u32(4);
    if (ifd + 2 > tn) {
        return 1;
    }
    const uint32_t count = u16(ifd);
    for (uint32_t i = 0; i < count; ++i) {
        const size_t e = ifd + 2 + size_t(i) * 12;
        if (e + 12 > tn) {
            break;
        }
        if (u16(e) == 0x0112 && u16(e + 2) == 3) {
            const uint32_t v = u16(e + 8);
            return v >= 1 && v <= 8 ? static_cast<int>(v) : 1;
        }
    }
    return 1;
}

// Applies EXIF orientation o to a w x h image (w, h updated).
void orient(std::vector<uint8_t>& px, int& w, int& h, int o) {
    if (o <= 1) {
        return;
    }
    const bool swap = o >= 5;
    const int nw = swap ? h : w, nh = swap ? w : h;
    std::vector<uint8_t> out(px.size());
    for (int y = 0; y < nh; ++y) {
        for (int x = 0; x < nw; ++x) {
            int sx, sy;   // source pixel of output (x, y)
            switch (o) {
                case 2: sx = w - 1 - x; sy = y; break;
                case 3: sx = w - 1 - x; sy = h - 1 - y; break;
                case 4: sx = x; sy = h - 1 - y; break;
                case 5: sx = y; sy = x; break;
                case 6: sx = y; sy = h - 1 - x; break;
                case 7: sx = w - 1 - y; sy = h - 1 - x; break;
                default: sx = w - 1 - y; sy = x; break;   // 8
            }
            out[size_t(y) * nw + x] = px[size_t(sy) * w + sx];
        }
    }
    px.swap(out);
    w = nw;
    h = nh;
}

ss_status decode_jpeg(const std::vector<uint8_t>& d, std::vector<uint8_t>& px,
                      int& w, int& h) {
    const size_t n = d.size();
    if (n < 4 || d[0] != 0xFF || d[1] != 0xD8) {
        return SS_ERR_INVALID_VALUE;
    }
    uint16_t qt[4][64];
    bool qt_defined[4] = {false, false, false, false};
    JpegHuff dc[4], ac[4];
    struct Comp {
        int id, hs, vs, tq;
    } comps[4];
    int ncomp = 0, width = 0, height = 0, restart = 0, orientation = 1;
    bool adobe_rgb = false;
    // The luma blocks' coefficients in natural order, before dequantisation
    // (a progressive file fills them over several scans).
    std::vector<int32_t> ycoef;
    bool progressive = false;
    int64_t eobrun = 0;
    size_t plane_w = 0;
    int y_blocks_w = 0, y_blocks_h = 0, hmax = 1, vmax = 1;
    bool y_done = false;
    size_t pos = 2;
    while (pos + 4 <= n) {
        if (d[pos] != 0xFF) {
            ++pos;   // stray bytes between segments
            continue;
        }
        const uint8_t m = d[pos + 1];
        if (m == 0xFF) {
            ++pos;
            continue;
        }
        pos += 2;
        if (m == 0xD9) {
            break;   // end of image
        }
        if ((m >= 0xD0 && m <= 0xD7) || m == 0x01) {
            continue;
        }
        const size_t len = (size_t(d[pos]) << 8) | d[pos + 1];
        if (len < 2 || pos + len > n) {
            return SS_ERR_INVALID_VALUE;
        }
        const uint8_t* seg = &d[pos + 2];
        const size_t sl = len - 2;
        if (m == 0xE1) {
            if (orientation == 1) {
                orientation = exif_orientation(seg, sl);
            }
        } else if (m == 0xEE) {
            // Adobe: transform 0 with three components means RGB samples.
            if (sl >= 12 && std::memcmp(seg, "Adobe", 5) == 0 && seg[11] == 0) {
                adobe_rgb = true;
            }
        } else if (m == 0xDB) {
            size_t q = 0;
            while (q < sl) {
                const int pq = seg[q] >> 4, tq = seg[q] & 15;
                if (tq > 3 || pq > 1 || q + 1 + 64 * (pq + 1) > sl) {
                    return SS_ERR_INVALID_VALUE;
                }
                for (int k = 0; k < 64; ++k) {
                    qt[tq][kZigzag[k]] = static_cast<uint16_t>(
                        pq ? (seg[q + 1 + 2 * k] << 8) | seg[q + 2 + 2 * k]
                           : seg[q + 1 + k]);
                }
                qt_defined[tq] = true;
                q += 1 + 64 * (pq + 1);
            }
        } else if (m == 0xC4) {
            size_t q = 0;
            while (q + 17 <= sl) {
                const int tc = seg[q] >> 4, th = seg[q] & 15;
                int total = 0;
                for (int k = 0; k < 16; ++k) {
                    total += seg[q + 1 + k];
                }
                if (tc > 1 || th > 3 || q + 17 + total > sl ||
                    !build_huff(seg + q + 1, seg + q + 17, total,
                                tc ? ac[th] : dc[th])) {
                    return SS_ERR_INVALID_VALUE;
                }
                q += 17 + total;
            }
        } else if (m == 0xDD) {
            if (sl < 2) {
                return SS_ERR_INVALID_VALUE;
            }
            restart = (seg[0] << 8) | seg[1];
        } else if (m == 0xC0 || m == 0xC1 || m == 0xC2) {
            progressive = m == 0xC2;
            if (sl < 6 || seg[0] != 8) {
                return SS_ERR_INVALID_VALUE;
            }
            height = (seg[1] << 8) | seg[2];
            width = (seg[3] << 8) | seg[4];
            ncomp = seg[5];
            if (width <= 0 || height <= 0 || (ncomp != 1 && ncomp != 3) ||
                sl < 6 + size_t(3) * ncomp) {
                return SS_ERR_INVALID_VALUE;   // DNL heights, CMYK refused
            }
            for (int i = 0; i < ncomp; ++i) {
                comps[i].id = seg[6 + 3 * i];
                comps[i].hs = seg[7 + 3 * i] >> 4;
                comps[i].vs = seg[7 + 3 * i] & 15;
                comps[i].tq = seg[8 + 3 * i];
                if (comps[i].hs < 1 || comps[i].hs > 4 || comps[i].vs < 1 ||
                    comps[i].vs > 4 || comps[i].tq > 3) {
                    return SS_ERR_INVALID_VALUE;
                }
                hmax = std::max(hmax, comps[i].hs);
                vmax = std::max(vmax, comps[i].vs);
            }
            // Gray output is the first component at full resolution.
            if (comps[0].hs != hmax || comps[0].vs != vmax ||
                (ncomp == 3 && comps[0].id == 'R' && comps[1].id == 'G' &&
                 comps[2].id == 'B')) {
                return SS_ERR_INVALID_VALUE;
            }
            const int mcu_w = 8 * hmax, mcu_h = 8 * vmax;
            const int mcus_x = (width + mcu_w - 1) / mcu_w;
            const int mcus_y = (height + mcu_h - 1) / mcu_h;
            y_blocks_w = mcus_x * hmax;
            y_blocks_h = mcus_y * vmax;
            plane_w = size_t(y_blocks_w) * 8;
            ycoef.assign(size_t(y_blocks_w) * size_t(y_blocks_h) * 64, 0);
        } else if ((m >= 0xC3 && m <= 0xCF) && m != 0xC4 && m != 0xC8 &&
                   m != 0xCC) {
            return SS_ERR_INVALID_VALUE;   // lossless, arithmetic
        } else if (m == 0xDA) {
            if (ycoef.empty() || sl < 1) {
                return SS_ERR_INVALID_VALUE;
            }
            const int ns = seg[0];
            if (ns < 1 || ns > ncomp || sl < 4 + size_t(2) * ns) {
                return SS_ERR_INVALID_VALUE;
            }
            int sc[4], std_dc[4], std_ac[4];
            bool has_y = false;
            for (int i = 0; i < ns; ++i) {
                const int cid = seg[1 + 2 * i];
                sc[i] = -1;
                for (int k = 0; k < ncomp; ++k) {
                    if (comps[k].id == cid) sc[i] = k;
                }
                std_dc[i] = seg[2 + 2 * i] >> 4;
                std_ac[i] = seg[2 + 2 * i] & 15;
                if (sc[i] < 0 || std_dc[i] > 3 || std_ac[i] > 3) {
                    return SS_ERR_INVALID_VALUE;
                }
                has_y = has_y || sc[i] == 0;
            }
            const int ss = seg[1 + 2 * ns], se = seg[2 + 2 * ns];
            const int ah = seg[3 + 2 * ns] >> 4, al = seg[3 + 2 * ns] & 15;
            if (!progressive) {
                if (ss != 0 || se != 63 || ah != 0 || al != 0) {
                    return SS_ERR_INVALID_VALUE;
                }
            } else if (se > 63 || ss > se || (ss == 0 && se != 0) ||
                       (ss > 0 && ns != 1) || al > 13 || ah > 13) {
                return SS_ERR_INVALID_VALUE;
            }
            pos += len;
            if (!has_y) {
                // Chroma only: skip the entropy-coded data.
                while (pos + 1 < n && !(d[pos] == 0xFF && d[pos + 1] != 0x00 &&
                                        !(d[pos + 1] >= 0xD0 && d[pos + 1] <= 0xD7))) {
                    ++pos;
                }
                continue;
            }
            const bool dc_scan = !progressive || ss == 0;
            const bool ac_scan = !progressive || ss > 0;
            for (int i = 0; i < ns; ++i) {
                if ((dc_scan && ah == 0 && !dc[std_dc[i]].defined) ||
                    (ac_scan && !ac[std_ac[i]].defined)) {
                    return SS_ERR_INVALID_VALUE;
                }
            }
            if (!qt_defined[comps[0].tq]) {
                return SS_ERR_INVALID_VALUE;
            }
            JpegBits br{d.data(), n, pos};
            int64_t pred[4] = {0, 0, 0, 0};   // 64-bit: hostile files
            eobrun = 0;
            // Units: interleaved MCUs, or the blocks of the one component.
            int units_x, units_y;
            if (ns > 1) {
                units_x = (width + 8 * hmax - 1) / (8 * hmax);
                units_y = (height + 8 * vmax - 1) / (8 * vmax);
            } else {
                const int cw = (width * comps[sc[0]].hs + hmax - 1) / hmax;
                const int ch = (height * comps[sc[0]].vs + vmax - 1) / vmax;
                units_x = (cw + 7) / 8;
                units_y = (ch + 7) / 8;
            }
            int32_t scratch[64];
            int64_t unit = 0;
            for (int uy = 0; uy < units_y; ++uy) {
                for (int ux = 0; ux < units_x; ++ux, ++unit) {
                    if (restart && unit > 0 && unit % restart == 0) {
                        if (br.short_data || !br.restart()) {
                            return SS_ERR_INVALID_VALUE;
                        }
                        pred[0] = pred[1] = pred[2] = pred[3] = 0;
                        eobrun = 0;
                    }
                    for (int i = 0; i < ns; ++i) {
                        const int k = sc[i];
                        const int bh = ns > 1 ? comps[k].hs : 1;
                        const int bv = ns > 1 ? comps[k].vs : 1;
                        for (int by = 0; by < bv; ++by) {
                            for (int bx = 0; bx < bh; ++bx) {
                                // The block's coefficients: a luma block of
                                // the image, else scratch (decoded to keep
                                // the bit stream in step, then dropped).
                                const int gx = ns > 1 ? ux * hmax + bx : ux;
                                const int gy = ns > 1 ? uy * vmax + by : uy;
                                int32_t* c = scratch;
                                if (k == 0 && gx < y_blocks_w && gy < y_blocks_h) {
                                    c = ycoef.data() +
                                        (size_t(gy) * y_blocks_w + gx) * 64;
                                }
                                if (c == scratch) {
                                    std::memset(scratch, 0, sizeof(scratch));
                                }
                                if (!decode_block(br, c, progressive, ss, se,
                                                  ah, al, dc[std_dc[i]],
                                                  ac[std_ac[i]], pred[i],
                                                  eobrun)) {
                                    return SS_ERR_INVALID_VALUE;
                                }
                            }
                        }
                    }
                }
            }
            if (br.short_data) {
                return SS_ERR_INVALID_VALUE;   // the data ended too early
            }
            y_done = true;
            // Continue after the entropy-coded segment.
            pos = br.pos;
            while (pos + 1 < n && !(d[pos] == 0xFF && d[pos + 1] != 0x00 &&
                                    !(d[pos + 1] >= 0xD0 && d[pos + 1] <= 0xD7))) {
                ++pos;
            }
            continue;
        }
        pos += len;
    }
    if (!y_done || (ncomp == 3 && adobe_rgb)) {
        return SS_ERR_INVALID_VALUE;
    }
    // Dequantise and inverse-transform every luma block.
    std::vector<uint8_t> plane(plane_w * size_t(y_blocks_h) * 8);
    const uint16_t* q = qt[comps[0].tq];
    int64_t block[64];
    for (int gy = 0; gy < y_blocks_h; ++gy) {
        for (int gx = 0; gx < y_blocks_w; ++gx) {
            const int32_t* c = ycoef.data() + (size_t(gy) * y_blocks_w + gx) * 64;
            for (int z = 0; z < 64; ++z) {
                block[z] = int64_t(c[z]) * q[z];
            }
            idct_islow(block, plane.data() + size_t(gy) * 8 * plane_w + size_t(gx) * 8,
                       plane_w);
        }
    }
    px.resize(size_t(width) * height);
    for (int y = 0; y < height; ++y) {
        std::memcpy(px.data() + size_t(y) * width, plane.data() + size_t(y) * plane_w,
                    size_t(width));
    }
    w = width;
    h = height;
    orient(px, w, h, orientation);
    return SS_OK;
}

// ---- TIFF ------------------------------------------------------------------
// First image of the file, chunky samples in strips or tiles, compression
// none, LZW, Deflate or PackBits, horizontal-difference predictor.  Gray as
// OpenCV returns it (each rule checked against OpenCV 4.13): 1-bit samples
// scale to 0 / 255; 16-bit samples keep their high byte; MinIsWhite is
// inverted; a gray image's alpha is ignored; 8-bit RGB and palette colours
// (16-bit map entries, high byte) take the BMP weights, and RGB with
// unassociated alpha is premultiplied first, (c a + 127) / 255; the
// Orientation tag is applied.  4-bit, 16-bit colour, planar, floating-point
// and JPEG-compressed images are refused.

uint32_t tiff_u16(const uint8_t* p, bool le) {
    return le ? le16(p) : (uint32_t(p[0]) << 8) | p[1];
}

uint32_t tiff_u32(const uint8_t* p, bool le) {
    return le ? le32(p)
              : (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) |
                    (uint32_t(p[2]) << 8) | p[3];
}

// TIFF LZW: MSB-first codes of 9..12 bits, 256 = clear, 257 = end, the code
// width growing one code early.
bool tiff_lzw(const uint8_t* in, size_t n, std::vector<uint8_t>& out,
              size_t want) {
    std::vector<uint16_t> prefix(4096);
    std::vector<uint8_t> suffix(4096), first(4096);
    std::vector<uint8_t> stack(4096);
    for (int i = 0; i < 256; ++i) {
        suffix[i] = first[i] = static_cast<uint8_t>(i);
    }
    int next = 258, width = 9, old = -1;
    uint32_t acc = 0;
    int have = 0;
    size_t pos = 0;
    out.clear();
    while (out.size() < want) {
        while (have < width) {
            if (pos >= n) {
                return out.size() >= want;
            }
            acc = (acc << 8) | in[pos++];
            have += 8;
        }
        const int code = static_cast<int>((acc >> (have - width)) &
                                          ((1u << width) - 1u));
        have -= width;
        if (code == 257) {
            break;
        }
        if (code == 256) {
            next = 258;
            width = 9;
            old = -1;
            continue;
        }
        int c = code, sp = 0;
        uint8_t firstc;
        if (old < 0) {
            if (code > 255) {
                return false;
            }
            out.push_back(static_cast<uint8_t>(code));
            old = code;
            continue;
        }
        if (code < next) {
            firstc = first[code];
        } else if (code == next) {
            firstc = first[old];
            stack[sp++] = firstc;
            c = old;
        } else {
            return false;
        }
        while (c > 255) {
            stack[sp++] = suffix[c];
            c = prefix[c];
        }
        stack[sp++] = static_cast<uint8_t>(c);
        while (sp) {
            out.push_back(stack[--sp]);
        }
        if (next < 4096) {
            prefix[next] = static_cast<uint16_t>(old);
            suffix[next] = firstc;
            first[next] = first[old];
            ++next;
        }
        if (next + 1 >= (1 << width) && width < 12) {
            ++width;
        }
        old = code;
    }
    return out.size() >= want;
}

bool tiff_packbits(const uint8_t* in, size_t n, std::vector<uint8_t>& out,
                   size_t want) {
    out.clear();
    size_t pos = 0;
    while (pos < n && out.size() < want) {
        const int c = static_cast<int8_t>(in[pos++]);
        if (c >= 0) {
            if (pos + c + 1 > n) return false;
            out.insert(out.end(), in + pos, in + pos + c + 1);
            pos += c + 1;
        } else if (c != -128) {
            if (pos >= n) return false;
            out.insert(out.end(), static_cast<size_t>(1 - c), in[pos++]);
        }
    }
    return out.size() >= want;
}

ss_status decode_tiff(const std::vector<uint8_t>& d, std::vector<uint8_t>& px,
                      int& w, int& h) {
    const size_t n = d.size();
    if (n < 8) return SS_ERR_INVALID_VALUE;
    const bool le = d[0] == 'I';
    if (tiff_u16(&d[2], le) != 42) return SS_ERR_INVALID_VALUE;
    const size_t ifd = tiff_u32(&d[4], le);
    if (ifd + 2 > n) return SS_ERR_INVALID_VALUE;
    const uint32_t count = tiff_u16(&d[ifd], le);
    if (ifd + 2 + size_t(count) * 12 > n) return SS_ERR_INVALID_VALUE;
    // Values of an entry (BYTE, SHORT or LONG).
    auto values = [&](size_t e, std::vector<uint32_t>& v) -> bool {
        const uint32_t type = tiff_u16(&d[e + 2], le);
        const uint32_t cnt = tiff_u32(&d[e + 4], le);
        const size_t size = type == 1 ? 1 : type == 3 ? 2 : type == 4 ? 4 : 0;
        if (!size || cnt > (1u << 24)) return false;
        size_t at = e + 8;
        if (size * cnt > 4) {
            at = tiff_u32(&d[e + 8], le);
            if (at + size * cnt > n) return false;
        }
        v.resize(cnt);
        for (uint32_t i = 0; i < cnt; ++i) {
            const uint8_t* q = &d[at + i * size];
            v[i] = size == 1 ? q[0] : size == 2 ? tiff_u16(q, le)
                                                : tiff_u32(q, le);
        }
        return true;
    };
    int64_t width = 0, height = 0;
    uint32_t bps = 1, comp = 1, phot = 1, spp = 1, planar = 1, pred = 1;
    uint32_t rps = 0xFFFFFFFFu, tile_w = 0, tile_h = 0, orientation = 1;
    uint32_t extra = 0xFFFFFFFFu, sample_format = 1;
    std::vector<uint32_t> offsets, counts, colormap, v;
    for (uint32_t k = 0; k < count; ++k) {
        const size_t e = ifd + 2 + size_t(k) * 12;
        const uint32_t tag = tiff_u16(&d[e], le);
        if (!values(e, v) || v.empty()) {
            continue;   // unknown types belong to tags not used here
        }
        switch (tag) {
            case 256: width = v[0]; break;
            case 257: height = v[0]; break;
            case 258: bps = v[0]; break;
            case 259: comp = v[0]; break;
            case 262: phot = v[0]; break;
            case 274: orientation = v[0]; break;
            case 277: spp = v[0]; break;
            case 278: rps = v[0]; break;
            case 284: planar = v[0]; break;
            case 317: pred = v[0]; break;
            case 320: colormap = v; break;
            case 322: tile_w = v[0]; break;
            case 323: tile_h = v[0]; break;
            case 338: extra = v[0]; break;
            case 339: sample_format = v[0]; break;
            case 273: case 324: offsets = v; break;
            case 279: case 325: counts = v; break;
            default: break;
        }
    }
    const bool gray = phot <= 1 && (spp == 1 || spp == 2);
    const bool rgb = phot == 2 && (spp == 3 || spp == 4) && bps == 8;
    const bool pal = phot == 3 && spp == 1 && bps == 8 &&
                     colormap.size() == 3 * 256;
    if (width <= 0 || height <= 0 || width * height > (int64_t(1) << 31) ||
        planar != 1 || sample_format != 1 || (pred != 1 && pred != 2) ||
        !(gray || rgb || pal) ||
        !(bps == 8 || (bps == 16 && gray) || (bps == 1 && spp == 1)) ||
        (comp != 1 && comp != 5 && comp != 8 && comp != 32946 &&
         comp != 32773) ||
        offsets.empty() || offsets.size() != counts.size()) {
        return SS_ERR_INVALID_VALUE;
    }
    const size_t W = size_t(width), H = size_t(height);
    const bool tiled = tile_w > 0 && tile_h > 0;
    const size_t bw = tiled ? tile_w : W;                 // block width
    const size_t bh = tiled ? tile_h : std::min<size_t>(rps, H);
    const size_t across = tiled ? (W + bw - 1) / bw : 1;
    const size_t down = (H + bh - 1) / bh;
    if (offsets.size() < across * down) return SS_ERR_INVALID_VALUE;
    const size_t row_bytes = (bw * spp * bps + 7) / 8;
    // All samples of the image, one row after another (row_out bytes).
    const size_t row_out = (W * spp * bps + 7) / 8;
    std::vector<uint8_t> img(row_out * H), buf;
    for (size_t by = 0; by < down; ++by) {
        for (size_t bx = 0; bx < across; ++bx) {
            const size_t k = by * across + bx;
            const size_t rows = tiled ? bh : std::min(bh, H - by * bh);
            const size_t want = row_bytes * rows;
            const size_t at = offsets[k], len = counts[k];
            if (at > n || len > n - at) return SS_ERR_INVALID_VALUE;
            const uint8_t* src = d.data() + at;
            bool ok = true;
            if (comp == 1) {
                ok = len >= want;
                buf.assign(src, src + std::min(len, want));
            } else if (comp == 5) {
                ok = tiff_lzw(src, len, buf, want);
            } else if (comp == 32773) {
                ok = tiff_packbits(src, len, buf, want);
            } else {
                buf.resize(want);
                uLongf out_len = static_cast<uLongf>(want);
                ok = uncompress(buf.data(), &out_len, src,
                                static_cast<uLong>(len)) == Z_OK &&
                     out_len == want;
            }
            if (!ok || buf.size() < want) return SS_ERR_INVALID_VALUE;
            for (size_t r = 0; r < rows; ++r) {
                uint8_t* row = buf.data() + r * row_bytes;
                if (pred == 2) {   // undo horizontal differencing
                    if (bps == 8) {
                        for (size_t i = spp; i < bw * spp; ++i) {
                            row[i] = static_cast<uint8_t>(row[i] + row[i - spp]);
                        }
                    } else if (bps == 16) {
                        for (size_t i = spp; i < bw * spp; ++i) {
                            const uint32_t a = tiff_u16(row + 2 * i, le) +
                                               tiff_u16(row + 2 * (i - spp), le);
                            row[2 * i + (le ? 0 : 1)] = static_cast<uint8_t>(a);
                            row[2 * i + (le ? 1 : 0)] =
                                static_cast<uint8_t>(a >> 8);
                        }
                    } else {
                        return SS_ERR_INVALID_VALUE;
                    }
                }
                const size_t y = by * bh + r;
                if (y >= H) break;
                // Columns of this block inside the image, in bytes.
                const size_t x0 = bx * bw;
                const size_t cols = std::min(bw, W - x0);
                const size_t o0 = (x0 * spp * bps) / 8;
                const size_t ob = (cols * spp * bps + 7) / 8;
                std::memcpy(img.data() + y * row_out + o0, row, ob);
            }
        }
    }
    px.resize(W * H);
    for (size_t y = 0; y < H; ++y) {
        const uint8_t* s = img.data() + y * row_out;
        uint8_t* o = px.data() + y * W;
        for (size_t x = 0; x < W; ++x) {
            uint32_t g;
            if (bps == 1) {
                g = ((s[x / 8] >> (7 - x % 8)) & 1u) ? 255u : 0u;
            } else if (gray) {
                g = bps == 16 ? tiff_u16(s + 2 * x * spp, le) >> 8
                              : s[x * spp];
            } else if (pal) {
                const uint32_t i = s[x];
                g = bgr_gray(colormap[512 + i] >> 8, colormap[256 + i] >> 8,
                             colormap[i] >> 8);
            } else {
                uint32_t r = s[x * spp], gg = s[x * spp + 1],
                         b = s[x * spp + 2];
                if (spp == 4 && extra == 2) {   // unassociated alpha
                    const uint32_t a = s[x * spp + 3];
                    r = (r * a + 127) / 255;
                    gg = (gg * a + 127) / 255;
                    b = (b * a + 127) / 255;
                }
                g = bgr_gray(static_cast<int>(b), static_cast<int>(gg),
                             static_cast<int>(r));
            }
            if (phot == 0) {
                g = 255u - g;   // MinIsWhite
            }
            o[x] = static_cast<uint8_t>(g);
        }
    }
    w = static_cast<int>(width);
    h = static_cast<int>(height);
    orient(px, w, h, static_cast<int>(orientation));
    return SS_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

ss_status read_image_impl(const char* path, uint8_t* pixels, size_t capacity,
                          int* width, int* height) {
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
    } else if (data.size() >= 2 && data[0] == 0xFF && data[1] == 0xD8) {
        st = decode_jpeg(data, px, w, h);
    } else if (data.size() >= 4 &&
               ((data[0] == 'I' && data[1] == 'I' && data[2] == 42 &&
                 data[3] == 0) ||
                (data[0] == 'M' && data[1] == 'M' && data[2] == 0 &&
                 data[3] == 42))) {
        st = decode_tiff(data, px, w, h);
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

}  // namespace

extern "C" {

ss_status ss_read_image(const char* path, uint8_t* pixels, size_t capacity,
                        int* width, int* height) {
    if (!path || !width || !height) {
        return SS_ERR_INVALID_VALUE;
    }
    // No exception crosses the C ABI: a file whose header claims more
    // pixels than the host can hold ends here.
    try {
        return read_image_impl(path, pixels, capacity, width, height);
    } catch (const std::bad_alloc&) {
        return SS_ERR_HOST_ALLOC;
    } catch (...) {
        return SS_ERR_INVALID_VALUE;
    }
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

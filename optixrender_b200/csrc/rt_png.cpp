// rt_png.cpp - PNG textures and PNG output without an image library.
//
// The reference loads textures with stb_image (core/src/Scene.cpp:181-189,
// forced to RGBA, flipped vertically so row 0 is the bottom).  This file
// decodes PNG files (ISO/IEC 15948) into the same layout and writes RGBA8
// frames as PNG.  The zlib stream (RFC 1950) carries DEFLATE data (RFC 1951),
// which is decoded with canonical Huffman codes: per code length the first
// code and the index of its first symbol, walked one bit at a time.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rt_image.h"

namespace rti {
namespace {

// ------------------------------------------------------------------ CRC-32 / Adler-32
uint32_t crc_table_entry(uint32_t c) {
    for (int k = 0; k < 8; k++) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
    return c;
}

uint32_t crc32(const uint8_t* p, size_t n, uint32_t crc = 0) {
    static uint32_t table[256];
    static bool ready = false;
    if (!ready) {
        for (uint32_t i = 0; i < 256; i++) table[i] = crc_table_entry(i);
        ready = true;
    }
    uint32_t c = crc ^ 0xFFFFFFFFu;
    for (size_t i = 0; i < n; i++) c = table[(c ^ p[i]) & 0xFFu] ^ (c >> 8);
    return c ^ 0xFFFFFFFFu;
}

uint32_t adler32(const uint8_t* p, size_t n) {
    uint32_t a = 1, b = 0;
    for (size_t i = 0; i < n; i++) {
        a = (a + p[i]) % 65521u;
        b = (b + a) % 65521u;
    }
    return (b << 16) | a;
}

// ------------------------------------------------------------------ DEFLATE
struct BitReader {
    const uint8_t* p;
    size_t n, pos = 0;  // byte position
    uint32_t bitbuf = 0;
    int bitcnt = 0;
    bool overrun = false;
    int bit() {
        if (bitcnt == 0) {
            if (pos >= n) {
                overrun = true;
                return 0;
            }
            bitbuf = p[pos++];
            bitcnt = 8;
        }
        int b = int(bitbuf & 1u);
        bitbuf >>= 1;
        bitcnt--;
        return b;
    }
    uint32_t bits(int k) {  // LSB first
        uint32_t v = 0;
        for (int i = 0; i < k; i++) v |= uint32_t(bit()) << i;
        return v;
    }
    void align() {
        bitcnt = 0;
        bitbuf = 0;
    }
};

// A canonical Huffman code: count of codes per length and the symbols in
// code order (RFC 1951 section 3.2.2).
struct Huffman {
    uint16_t count[16];
    std::vector<uint16_t> symbol;
    // returns false for an over-subscribed code; incomplete codes are allowed
    // (a single distance code is legal)
    bool build(const uint8_t* lengths, int n) {
        std::memset(count, 0, sizeof(count));
        for (int s = 0; s < n; s++) count[lengths[s]]++;
        count[0] = 0;
        int left = 1;
        for (int len = 1; len < 16; len++) {
            left <<= 1;
            left -= count[len];
            if (left < 0) return false;
        }
        uint16_t offs[16];
        offs[1] = 0;
        for (int len = 1; len < 15; len++) offs[len + 1] = uint16_t(offs[len] + count[len]);
        symbol.assign(size_t(n), 0);
        for (int s = 0; s < n; s++)
            if (lengths[s]) symbol[offs[lengths[s]]++] = uint16_t(s);
        return true;
    }
    int decode(BitReader& br) const {
        int code = 0, first = 0, index = 0;
        for (int len = 1; len < 16; len++) {
            code |= br.bit();
            const int c = count[len];
            if (code - first < c) return symbol[size_t(index + code - first)];
            index += c;
            first = (first + c) << 1;
            code <<= 1;
            if (br.overrun) return -1;
        }
        return -1;
    }
};

const uint16_t kLenBase[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                               31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
const uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t kDistBase[30] = {1,   2,   3,   4,   5,   7,    9,    13,   17,   25,   33,   49,   65,    97,    129,
                                193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
const uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

bool inflate_block(BitReader& br, const Huffman& lit, const Huffman& dist, std::vector<uint8_t>& out, size_t limit,
                   std::string& err) {
    while (true) {
        int sym = lit.decode(br);
        if (sym < 0) {
            err = "bad literal/length code";
            return false;
        }
        if (sym < 256) {
            if (out.size() >= limit) {
                err = "image data longer than expected";
                return false;
            }
            out.push_back(uint8_t(sym));
            continue;
        }
        if (sym == 256) return true;
        sym -= 257;
        if (sym >= 29) {
            err = "bad length symbol";
            return false;
        }
        const size_t len = kLenBase[sym] + br.bits(kLenExtra[sym]);
        const int ds = dist.decode(br);
        if (ds < 0 || ds >= 30) {
            err = "bad distance code";
            return false;
        }
        const size_t d = kDistBase[ds] + br.bits(kDistExtra[ds]);
        if (d > out.size()) {
            err = "distance before the start of the data";
            return false;
        }
        if (out.size() + len > limit) {
            err = "image data longer than expected";
            return false;
        }
        const size_t from = out.size() - d;
        for (size_t i = 0; i < len; i++) out.push_back(out[from + i]);  // copies may overlap
        if (br.overrun) {
            err = "truncated compressed data";
            return false;
        }
    }
}

bool dynamic_tables(BitReader& br, Huffman& lit, Huffman& dist, std::string& err) {
    const int hlit = int(br.bits(5)) + 257, hdist = int(br.bits(5)) + 1, hclen = int(br.bits(4)) + 4;
    static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
    uint8_t cl[19] = {0};
    for (int i = 0; i < hclen; i++) cl[order[i]] = uint8_t(br.bits(3));
    Huffman clh;
    if (!clh.build(cl, 19)) {
        err = "bad code-length code";
        return false;
    }
    uint8_t lengths[320] = {0};
    int i = 0;
    while (i < hlit + hdist) {
        int sym = clh.decode(br);
        if (sym < 0) {
            err = "bad code-length symbol";
            return false;
        }
        if (sym < 16) {
            lengths[i++] = uint8_t(sym);
            continue;
        }
        uint8_t v = 0;
        int rep;
        if (sym == 16) {
            if (i == 0) {
                err = "repeat with no previous length";
                return false;
            }
            v = lengths[i - 1];
            rep = 3 + int(br.bits(2));
        } else if (sym == 17) {
            rep = 3 + int(br.bits(3));
        } else {
            rep = 11 + int(br.bits(7));
        }
        if (i + rep > hlit + hdist) {
            err = "code lengths overflow";
            return false;
        }
        while (rep--) lengths[i++] = v;
    }
    if (lengths[256] == 0) {
        err = "no end-of-block code";
        return false;
    }
    if (!lit.build(lengths, hlit) || !dist.build(lengths + hlit, hdist)) {
        err = "bad literal/length or distance code";
        return false;
    }
    return true;
}

}  // namespace

bool zlib_inflate(const uint8_t* src, size_t n, std::vector<uint8_t>& out, size_t expected, std::string& err) {
    if (n < 6) {
        err = "truncated zlib stream";
        return false;
    }
    const uint8_t cmf = src[0], flg = src[1];
    if ((cmf & 0x0Fu) != 8 || (cmf >> 4) > 7 || ((uint32_t(cmf) << 8) | flg) % 31u != 0 || (flg & 0x20u)) {
        err = "not a zlib deflate stream";
        return false;
    }
    BitReader br{src + 2, n - 2};
    out.clear();
    out.reserve(expected);
    Huffman fixed_lit, fixed_dist;
    {
        uint8_t l[288];
        for (int i = 0; i < 144; i++) l[i] = 8;
        for (int i = 144; i < 256; i++) l[i] = 9;
        for (int i = 256; i < 280; i++) l[i] = 7;
        for (int i = 280; i < 288; i++) l[i] = 8;
        fixed_lit.build(l, 288);
        uint8_t d[30];
        for (int i = 0; i < 30; i++) d[i] = 5;
        fixed_dist.build(d, 30);
    }
    bool last = false;
    while (!last) {
        last = br.bit() != 0;
        const uint32_t type = br.bits(2);
        if (type == 0) {  // stored
            br.align();
            if (br.pos + 4 > br.n) {
                err = "truncated stored block";
                return false;
            }
            const uint32_t len = uint32_t(br.p[br.pos]) | (uint32_t(br.p[br.pos + 1]) << 8);
            const uint32_t nlen = uint32_t(br.p[br.pos + 2]) | (uint32_t(br.p[br.pos + 3]) << 8);
            br.pos += 4;
            if ((len ^ 0xFFFFu) != nlen || br.pos + len > br.n || out.size() + len > expected) {
                err = "bad stored block";
                return false;
            }
            out.insert(out.end(), br.p + br.pos, br.p + br.pos + len);
            br.pos += len;
        } else if (type == 1) {
            if (!inflate_block(br, fixed_lit, fixed_dist, out, expected, err)) return false;
        } else if (type == 2) {
            Huffman lit, dist;
            if (!dynamic_tables(br, lit, dist, err)) return false;
            if (!inflate_block(br, lit, dist, out, expected, err)) return false;
        } else {
            err = "bad deflate block type";
            return false;
        }
        if (br.overrun) {
            err = "truncated compressed data";
            return false;
        }
    }
    br.align();
    if (br.pos + 4 <= br.n) {
        const uint32_t want = (uint32_t(br.p[br.pos]) << 24) | (uint32_t(br.p[br.pos + 1]) << 16) |
                              (uint32_t(br.p[br.pos + 2]) << 8) | uint32_t(br.p[br.pos + 3]);
        if (want != adler32(out.data(), out.size())) {
            err = "zlib checksum mismatch";
            return false;
        }
    }
    return true;
}

namespace {

uint32_t be32(const uint8_t* p) { return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3]; }

int paeth(int a, int b, int c) {
    const int p = a + b - c, pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p, pc = p > c ? p - c : c - p;
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

}  // namespace

bool read_png(const std::string& d, std::vector<uint8_t>& rgba, int& w, int& h, std::string& err) {
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    const uint8_t* p = reinterpret_cast<const uint8_t*>(d.data());
    const size_t n = d.size();
    if (n < 8 || std::memcmp(p, sig, 8) != 0) {
        err = "not a PNG file";
        return false;
    }
    size_t pos = 8;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, palette, trns;
    bool have_ihdr = false, have_iend = false;
    while (pos + 12 <= n && !have_iend) {
        const uint32_t len = be32(p + pos);
        if (len > n - pos - 12) {
            err = "truncated chunk";
            return false;
        }
        const uint8_t* type = p + pos + 4;
        const uint8_t* data = p + pos + 8;
        if (crc32(type, size_t(len) + 4) != be32(data + len)) {
            err = "chunk CRC mismatch";
            return false;
        }
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len != 13) {
                err = "bad IHDR";
                return false;
            }
            w = int(be32(data));
            h = int(be32(data + 4));
            depth = data[8];
            ctype = data[9];
            interlace = data[12];
            if (data[10] != 0 || data[11] != 0) {
                err = "unknown compression or filter method";
                return false;
            }
            have_ihdr = true;
        } else if (!std::memcmp(type, "PLTE", 4)) {
            palette.assign(data, data + len);
        } else if (!std::memcmp(type, "tRNS", 4)) {
            trns.assign(data, data + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            have_iend = true;
        } else if (!(type[0] & 0x20u)) {
            err = "unknown critical chunk";
            return false;
        }
        pos += size_t(len) + 12;
    }
    if (!have_ihdr || idat.empty()) {
        err = "missing IHDR or IDAT";
        return false;
    }
    if (w <= 0 || h <= 0 || int64_t(w) * h > (int64_t(1) << 28)) {
        err = "bad image size";
        return false;
    }
    if (interlace != 0) {
        err = "interlaced PNG is not supported";
        return false;
    }
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: err = "bad colour type"; return false;
    }
    const bool depth_ok = depth == 8 || (depth == 16 && ctype != 3) ||
                          ((depth == 1 || depth == 2 || depth == 4) && (ctype == 0 || ctype == 3));
    if (!depth_ok) {
        err = "unsupported bit depth";
        return false;
    }
    if (ctype == 3 && (palette.empty() || palette.size() % 3)) {
        err = "palette image without a valid PLTE";
        return false;
    }
    const size_t bits_pp = size_t(channels) * size_t(depth);
    const size_t stride = (size_t(w) * bits_pp + 7) / 8;
    const size_t bpp = (bits_pp + 7) / 8;  // filter unit in bytes
    std::vector<uint8_t> raw;
    if (!zlib_inflate(idat.data(), idat.size(), raw, (stride + 1) * size_t(h), err)) return false;
    if (raw.size() != (stride + 1) * size_t(h)) {
        err = "image data shorter than expected";
        return false;
    }
    // undo the per-row filters in place (the previous row is already decoded)
    for (int y = 0; y < h; y++) {
        uint8_t* row = raw.data() + size_t(y) * (stride + 1);
        const uint8_t f = row[0];
        uint8_t* cur = row + 1;
        const uint8_t* prev = y > 0 ? raw.data() + size_t(y - 1) * (stride + 1) + 1 : nullptr;
        for (size_t i = 0; i < stride; i++) {
            const int a = i >= bpp ? cur[i - bpp] : 0, b = prev ? prev[i] : 0, c = (prev && i >= bpp) ? prev[i - bpp] : 0;
            int v;
            switch (f) {
                case 0: v = 0; break;
                case 1: v = a; break;
                case 2: v = b; break;
                case 3: v = (a + b) >> 1; break;
                case 4: v = paeth(a, b, c); break;
                default: err = "bad filter type"; return false;
            }
            cur[i] = uint8_t(cur[i] + v);
        }
    }
    // to RGBA8, row 0 = bottom of the picture (stbi's vertical flip)
    rgba.assign(size_t(w) * size_t(h) * 4, 255);
    auto sample = [&](const uint8_t* row, int x, int ch) -> int {  // value of channel ch, scaled to 8 bits
        if (depth == 8) return row[size_t(x) * channels + ch];
        if (depth == 16) return row[(size_t(x) * channels + ch) * 2];
        const size_t bit = size_t(x) * depth;
        const int v = (row[bit >> 3] >> (8 - depth - int(bit & 7))) & ((1 << depth) - 1);
        return ctype == 3 ? v : v * 255 / ((1 << depth) - 1);
    };
    auto raw16 = [&](const uint8_t* row, int x, int ch) -> int {
        return depth == 16 ? (row[(size_t(x) * channels + ch) * 2] << 8) | row[(size_t(x) * channels + ch) * 2 + 1]
                           : -1;
    };
    for (int y = 0; y < h; y++) {
        const uint8_t* row = raw.data() + size_t(y) * (stride + 1) + 1;
        uint8_t* dst = rgba.data() + size_t(h - 1 - y) * size_t(w) * 4;
        for (int x = 0; x < w; x++) {
            uint8_t* o = dst + size_t(x) * 4;
            if (ctype == 3) {
                const int idx = sample(row, x, 0);
                if (size_t(idx) * 3 + 2 >= palette.size()) {
                    err = "palette index out of range";
                    return false;
                }
                o[0] = palette[size_t(idx) * 3];
                o[1] = palette[size_t(idx) * 3 + 1];
                o[2] = palette[size_t(idx) * 3 + 2];
                o[3] = size_t(idx) < trns.size() ? trns[size_t(idx)] : 255;
            } else if (ctype == 0 || ctype == 4) {
                const int g = sample(row, x, 0);
                o[0] = o[1] = o[2] = uint8_t(g);
                if (ctype == 4) {
                    o[3] = uint8_t(sample(row, x, 1));
                } else if (trns.size() >= 2) {  // one grey value is transparent
                    const int key = (trns[0] << 8) | trns[1];
                    const int v = depth == 16 ? raw16(row, x, 0) : (depth == 8 ? g : (g * ((1 << depth) - 1) + 127) / 255);
                    if (v == key) o[3] = 0;
                }
            } else {
                o[0] = uint8_t(sample(row, x, 0));
                o[1] = uint8_t(sample(row, x, 1));
                o[2] = uint8_t(sample(row, x, 2));
                if (ctype == 6) {
                    o[3] = uint8_t(sample(row, x, 3));
                } else if (trns.size() >= 6) {  // one colour is transparent
                    bool match = true;
                    for (int ch = 0; ch < 3; ch++) {
                        const int key = (trns[size_t(2 * ch)] << 8) | trns[size_t(2 * ch + 1)];
                        const int v = depth == 16 ? raw16(row, x, ch) : sample(row, x, ch);
                        match = match && v == key;
                    }
                    if (match) o[3] = 0;
                }
            }
        }
    }
    return true;
}

namespace {
void put32(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back(uint8_t(x >> 24));
    v.push_back(uint8_t(x >> 16));
    v.push_back(uint8_t(x >> 8));
    v.push_back(uint8_t(x));
}
void chunk(std::vector<uint8_t>& file, const char* type, const std::vector<uint8_t>& data) {
    put32(file, uint32_t(data.size()));
    const size_t start = file.size();
    file.insert(file.end(), type, type + 4);
    file.insert(file.end(), data.begin(), data.end());
    put32(file, crc32(file.data() + start, data.size() + 4));
}
}  // namespace

bool write_png(const std::string& path, const uint32_t* rgba8, int w, int h, std::string& err) {
    if (!rgba8 || w <= 0 || h <= 0) {
        err = "bad image";
        return false;
    }
    // filter type 0 rows, top row first (row 0 of the frame is the bottom)
    const size_t stride = size_t(w) * 4 + 1;
    std::vector<uint8_t> raw(stride * size_t(h));
    for (int y = 0; y < h; y++) {
        uint8_t* row = raw.data() + size_t(y) * stride;
        row[0] = 0;
        std::memcpy(row + 1, rgba8 + size_t(h - 1 - y) * size_t(w), size_t(w) * 4);
    }
    // zlib stream of stored blocks (no compression)
    std::vector<uint8_t> z = {0x78, 0x01};
    for (size_t off = 0; off < raw.size() || off == 0;) {
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        const bool last = off + len == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back(uint8_t(len));
        z.push_back(uint8_t(len >> 8));
        z.push_back(uint8_t(~len));
        z.push_back(uint8_t(~len >> 8));
        z.insert(z.end(), raw.begin() + long(off), raw.begin() + long(off + len));
        off += len;
        if (last) break;
    }
    put32(z, adler32(raw.data(), raw.size()));
    std::vector<uint8_t> file = {137, 80, 78, 71, 13, 10, 26, 10};
    std::vector<uint8_t> ihdr;
    put32(ihdr, uint32_t(w));
    put32(ihdr, uint32_t(h));
    ihdr.insert(ihdr.end(), {8, 6, 0, 0, 0});
    chunk(file, "IHDR", ihdr);
    chunk(file, "IDAT", z);
    chunk(file, "IEND", {});
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        err = "could not open " + path;
        return false;
    }
    const bool ok = std::fwrite(file.data(), 1, file.size(), f) == file.size();
    return std::fclose(f) == 0 && ok;
}

}  // namespace rti
